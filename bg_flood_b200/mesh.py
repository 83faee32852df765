"""Block-uniform quadtree (BUQ) helpers for building models from regular grids.

The BUQ layout is the reference's: per block an 18x18 tile (16x16 cells and a
one-cell halo), cell (i, j) of block ib at ``(i+1) + (j+1)*18 + ib*324``
(memloc, src/MemManagement.cu:37-40).  Neighbour tables are returned as an
``(nblk, 8)`` array in the order LeftBot, LeftTop, RightBot, RightTop, BotLeft,
BotRight, TopLeft, TopRight.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._native import lib

__all__ = ["Mesh", "uniform_mesh", "grid_to_buq", "buq_to_grid", "fill_halo", "boundary_segments",
           "NBR_ORDER"]

NBR_ORDER = ("LeftBot", "LeftTop", "RightBot", "RightTop", "BotLeft", "BotRight", "TopLeft", "TopRight")


@dataclass
class Mesh:
    nbx: int
    nby: int
    dx: float
    nblk: int
    level: np.ndarray   # (nblk,) int32
    nbr: np.ndarray     # (nblk, 8) int32
    xo: np.ndarray      # (nblk,) block origin (first cell centre) relative to the domain origin
    yo: np.ndarray
    bx: np.ndarray      # (nblk,) block column / row in the level-0 grid
    by: np.ndarray

    @property
    def active(self) -> np.ndarray:
        return np.arange(self.nblk, dtype=np.int32)


def uniform_mesh(nx: int, ny: int, dx: float, present: np.ndarray | None = None, doubleprecision: bool = False) -> Mesh:
    """Uniform level-0 mesh of nx*ny cells (multiples of 16), as InitBlockxoyo and
    InitBlockneighbours build it (src/Mesh.cu:257-433).  ``present`` (nby, nbx) masks
    out blocks (the reference drops blocks whose cells are all above ``mask``)."""
    if nx % 16 or ny % 16:
        raise ValueError("nx and ny must be multiples of 16")
    nbx, nby = nx // 16, ny // 16
    nmax = nbx * nby
    pres = None
    if present is not None:
        pres = np.ascontiguousarray(present, dtype=np.uint8).reshape(-1)
    nblk = ctypes.c_int(0)
    level = np.zeros(nmax, np.int32)
    nbr = np.zeros(nmax * 8, np.int32)
    xo = np.zeros(nmax)
    yo = np.zeros(nmax)
    rc = lib().bgf_mesh_uniform(nbx, nby, float(dx), pres.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if pres is not None else None,
                                ctypes.byref(nblk), level.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                nbr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                xo.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                yo.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1 if doubleprecision else 0)
    if rc != 0:
        raise RuntimeError(f"bgf_mesh_uniform failed ({rc})")
    n = nblk.value
    idx = np.flatnonzero(pres) if pres is not None else np.arange(nmax)
    return Mesh(nbx, nby, dx, n, level[:n].copy(), nbr[: 8 * n].reshape(n, 8).copy(), xo[:n].copy(), yo[:n].copy(),
                (idx % nbx).astype(np.int32), (idx // nbx).astype(np.int32))


def grid_to_buq(a: np.ndarray, mesh: Mesh, dtype=np.float64) -> np.ndarray:
    """Row-major (ny, nx) cell array -> (nblk, 18, 18) BUQ tiles (halo left at 0)."""
    out = np.zeros((mesh.nblk, 18, 18), dtype)
    t = a.reshape(mesh.nby, 16, mesh.nbx, 16).transpose(0, 2, 1, 3)  # (by, bx, j, i)
    out[:, 1:17, 1:17] = t[mesh.by, mesh.bx]
    return out


def buq_to_grid(b: np.ndarray, mesh: Mesh, fill=np.nan) -> np.ndarray:
    """(nblk, 18, 18) tiles -> (ny, nx) cell array (cells of absent blocks = fill)."""
    b = np.asarray(b).reshape(-1, 18, 18)
    out = np.full((mesh.nby, mesh.nbx, 16, 16), fill, dtype=b.dtype)
    out[mesh.by, mesh.bx] = b[: mesh.nblk, 1:17, 1:17]
    return out.transpose(0, 2, 1, 3).reshape(mesh.nby * 16, mesh.nbx * 16)


def fill_halo(b: np.ndarray, mesh: Mesh) -> np.ndarray:
    """Halo fill of one BUQ field on a single-level mesh, as fillHaloC does
    (src/Halo.cu:43-51 with fillLeft/Right/Top/Bot, :2083-2286): a same-level
    neighbour's edge row/column, or the block's own edge at the domain boundary.
    Corner halo cells are left as they are, like the reference."""
    b = np.array(b, copy=True).reshape(-1, 18, 18)
    n = mesh.nblk
    ib = np.arange(n)
    L, R, B, T = mesh.nbr[:, 0], mesh.nbr[:, 2], mesh.nbr[:, 4], mesh.nbr[:, 6]
    if np.any(mesh.level[L] != mesh.level) or np.any(mesh.level[R] != mesh.level):
        raise NotImplementedError("cross-level halos are not handled by this helper")
    left = np.where((L == ib)[:, None], b[ib, 1:17, 1], b[L, 1:17, 16])
    right = np.where((R == ib)[:, None], b[ib, 1:17, 16], b[R, 1:17, 1])
    top = np.where((T == ib)[:, None], b[ib, 16, 1:17], b[T, 1, 1:17])
    bot = np.where((B == ib)[:, None], b[ib, 1, 1:17], b[B, 16, 1:17])
    b[:n, 1:17, 0] = left
    b[:n, 1:17, 17] = right
    b[:n, 17, 1:17] = top
    b[:n, 0, 1:17] = bot
    return b


def _side_polygon(side: str, xo: float, yo: float, xmax: float, ymax: float, eps: float):
    # readbndpolysegment (src/ReadForcing.cu:722-870): thin rectangles along the sides
    if side == "left":
        return (xo - eps, xo + eps, yo, ymax)
    if side == "right":
        return (xmax - eps, xmax + eps, yo, ymax)
    if side == "bot":
        return (xo, xmax, yo - eps, yo + eps)
    if side == "top":
        return (xo, xmax, ymax - eps, ymax + eps)
    return (xo - eps, xmax + eps, yo - eps, ymax + eps)  # "all"


def boundary_segments(mesh: Mesh, segments: list, aoibnd: int, xo: float = 0.0, yo: float = 0.0):
    """Assigns the domain-edge blocks to boundary segments as Calcbndblks /
    Findbndblks do (src/InitialConditions.cu:1160-1300): a block with any side on
    the domain edge belongs to the last declared segment whose polygon holds one of
    its corners (blockinpoly, src/Poly.cu:443-503), otherwise to the remainder
    segment of type ``aoibnd`` (src/ReadInput.cu:1338-1354).  Returns a list of
    (type, times, levels, [left, right, top, bot] block lists) in application order."""
    n = mesh.nblk
    ib = np.arange(n)
    nb = mesh.nbr
    edge = np.any(nb == ib[:, None], axis=1)
    xmax = xo + mesh.nbx * 16 * mesh.dx
    ymax = yo + mesh.nby * 16 * mesh.dx
    owner = np.full(n, len(segments), np.int64)
    for s, seg in enumerate(segments):
        x0, x1, y0, y1 = _side_polygon(seg.side, xo, yo, xmax, ymax, mesh.dx)
        for b in np.flatnonzero(edge):
            lev_dx = mesh.dx / (1 << int(mesh.level[b])) if mesh.level[b] >= 0 else mesh.dx * (1 << -int(mesh.level[b]))
            bx0 = xo + mesh.xo[b]
            by0 = yo + mesh.yo[b]
            corners = [(bx0, by0), (bx0 + 16 * lev_dx, by0), (bx0, by0 + 16 * lev_dx), (bx0 + 16 * lev_dx, by0 + 16 * lev_dx)]
            if any(x0 <= cx <= x1 and y0 <= cy <= y1 for cx, cy in corners):
                owner[b] = s
    out = []
    specs = list(segments) + [None]
    for s, seg in enumerate(specs):
        typ = aoibnd if seg is None else seg.type
        times = [] if seg is None else list(seg.times)
        levels = [] if seg is None else list(seg.levels)
        mine = edge & (owner == s)
        sides = [
            np.flatnonzero(mine & ((nb[:, 0] == ib) | (nb[:, 1] == ib))),
            np.flatnonzero(mine & ((nb[:, 2] == ib) | (nb[:, 3] == ib))),
            np.flatnonzero(mine & ((nb[:, 6] == ib) | (nb[:, 7] == ib))),
            np.flatnonzero(mine & ((nb[:, 4] == ib) | (nb[:, 5] == ib))),
        ]
        out.append((typ, times, levels, [x.astype(np.int32) for x in sides]))
    return out
