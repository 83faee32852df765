"""Python host side of the flow-step library: a thin wrapper over the C ABI.

``FlowB200`` owns one library handle (device memory for the BUQ state of one
scenario).  Its methods map one-to-one onto the C entry points of
include/bg_flood_b200.h, which in turn stand in for the reference's SetupGPU /
CopytoGPU and FlowGPU (src/Setup_GPU.cu:15-375, src/FlowGPU.cu:14-315).
``build_model`` assembles a handle from regular-grid arrays the way the
reference's own tests set up a model in memory (src/Testing.cu:418-588).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from ._native import lib
from .mesh import Mesh, boundary_segments, fill_halo, grid_to_buq, uniform_mesh
from .params import Param

__all__ = ["FlowB200", "BGFError", "Loop", "build_model", "CBlockP", "CEvolving", "CLoop"]


class BGFError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().bgf_strerror(status).decode()
        last = lib().bgf_last_error().decode()
        super().__init__(f"{where}: {msg} (status {status}){': ' + last if last else ''}")
        self.status = status


class CLoop(ctypes.Structure):
    _fields_ = [("nextoutputtime", ctypes.c_double), ("dt", ctypes.c_double), ("dtmax", ctypes.c_double),
                ("totaltime", ctypes.c_double)]


class CBlockP(ctypes.Structure):
    _fields_ = [("nblk", ctypes.c_int), ("active", ctypes.c_void_p), ("level", ctypes.c_void_p)] + \
        [(n, ctypes.c_void_p) for n in ("BotLeft", "BotRight", "TopLeft", "TopRight", "LeftBot", "LeftTop",
                                        "RightBot", "RightTop", "xo", "yo")]


class CAdaptParam(ctypes.Structure):
    _fields_ = [("criterion", ctypes.c_int), ("var", ctypes.c_int), ("arg1", ctypes.c_double),
                ("arg2", ctypes.c_double), ("maxiteration", ctypes.c_int), ("allow_coarsen", ctypes.c_int)]


class CEvolving(ctypes.Structure):
    _fields_ = [("zs", ctypes.c_void_p), ("h", ctypes.c_void_p), ("u", ctypes.c_void_p), ("v", ctypes.c_void_p)]


@dataclass
class Loop:
    """Reference Loop<T> members the step uses (src/Arrays.h:359-404)."""
    totaltime: float = 0.0
    dt: float = 0.0
    dtmax: float = 0.0
    nextoutputtime: float = 0.0

    def to_c(self) -> CLoop:
        return CLoop(self.nextoutputtime, self.dt, self.dtmax, self.totaltime)

    def from_c(self, c: CLoop) -> None:
        self.nextoutputtime, self.dt, self.dtmax, self.totaltime = c.nextoutputtime, c.dt, c.dtmax, c.totaltime


def _check(rc: int, where: str) -> None:
    if rc != 0:
        raise BGFError(rc, where)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class FlowB200:
    """One scenario on one GPU through the C ABI."""

    def __init__(self, param: Param, nblkmem: int, stream: int | None = None):
        self.param = param
        # field arrays at the C boundary: double with doubleprecision or split precision
        self.dtype = np.float64 if (param.doubleprecision or getattr(param, "splitprecision", 0)) else np.float32
        self.dev_dtype = np.float64 if param.doubleprecision else np.float32
        self.nblkmem = int(nblkmem)
        self._cparam = param.to_c()
        h = ctypes.c_void_p()
        _check(lib().bgf_create(ctypes.byref(self._cparam), self.nblkmem, ctypes.c_void_p(stream) if stream else None,
                                ctypes.byref(h)), "bgf_create")
        self.handle = h
        self._keep = []

    def close(self) -> None:
        if self.handle:
            lib().bgf_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nblk(self) -> int:
        """Active blocks of the current mesh."""
        n = ctypes.c_int(0)
        _check(lib().bgf_get_blocks(self.handle, ctypes.byref(n), None, None, None, None, None), "bgf_get_blocks")
        return n.value

    # -- set-up -------------------------------------------------------------------
    def set_blocks(self, active: np.ndarray, level: np.ndarray, nbr: np.ndarray, xo=None, yo=None) -> None:
        """Block tables; nbr is (nblkmem, 8) in LeftBot, LeftTop, RightBot, RightTop,
        BotLeft, BotRight, TopLeft, TopRight order."""
        active = np.ascontiguousarray(active, np.int32)
        lv = np.zeros(self.nblkmem, np.int32)
        lv[: len(level)] = level
        nb = np.zeros((self.nblkmem, 8), np.int32)
        nb[: len(nbr)] = nbr
        cols = [np.ascontiguousarray(nb[:, k]) for k in range(8)]
        fx = np.zeros(self.nblkmem, self.dtype)
        fy = np.zeros(self.nblkmem, self.dtype)
        if xo is not None:
            fx[: len(xo)] = xo
            fy[: len(yo)] = yo
        b = CBlockP()
        b.nblk = len(active)
        b.active, b.level = _ptr(active), _ptr(lv)
        b.LeftBot, b.LeftTop, b.RightBot, b.RightTop = (_ptr(c) for c in cols[:4])
        b.BotLeft, b.BotRight, b.TopLeft, b.TopRight = (_ptr(c) for c in cols[4:])
        b.xo, b.yo = _ptr(fx), _ptr(fy)
        self._keep = [active, lv, cols, fx, fy]
        _check(lib().bgf_set_blocks(self.handle, ctypes.byref(b)), "bgf_set_blocks")

    def set_bed(self, zb: np.ndarray, dzbdx=None, dzbdy=None, cf=None, activeCell=None) -> None:
        """BUQ (nblkmem, 18, 18) arrays; zb with its halo filled."""
        conv = lambda a: None if a is None else np.ascontiguousarray(a, self.dtype)
        zb, dzbdx, dzbdy, cf = conv(zb), conv(dzbdx), conv(dzbdy), conv(cf)
        ac = None if activeCell is None else np.ascontiguousarray(activeCell, np.int32)
        _check(lib().bgf_set_bed(self.handle, _ptr(zb), _ptr(dzbdx), _ptr(dzbdy), _ptr(cf),
                                 None if ac is None else ac.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), "bgf_set_bed")

    def add_segment(self, typ: int, times, levels, sides) -> None:
        t = np.ascontiguousarray(times, np.float64)
        w = np.ascontiguousarray(levels, np.float64)
        arrs = [np.ascontiguousarray(s, np.int32) for s in sides]
        cnt = (ctypes.c_int * 4)(*[len(a) for a in arrs])
        ptrs = (ctypes.POINTER(ctypes.c_int) * 4)(*[a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) for a in arrs])
        _check(lib().bgf_add_bnd_segment(self.handle, int(typ), len(t), t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cnt, ptrs), "bgf_add_bnd_segment")

    def set_rain(self, times, rates_mmh) -> None:
        t = np.ascontiguousarray(times, np.float64)
        r = np.ascontiguousarray(rates_mmh, np.float64)
        _check(lib().bgf_set_rain_series(self.handle, len(t), t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "bgf_set_rain_series")

    def set_rain_map(self, xo: float, yo: float, dx: float, dy: float, to: float, dt: float, frames) -> None:
        """Gridded rain (mm/h): frames (nt, ny, nx) of nodes from (xo, yo), frame k at
        time to + k*dt."""
        fr = np.ascontiguousarray(frames, np.float32)
        nt, ny, nx = fr.shape
        _check(lib().bgf_set_rain_map(self.handle, nx, ny, float(xo), float(yo), float(dx), float(dy), nt,
                                      float(to), float(dt), fr.ctypes.data), "bgf_set_rain_map")
        self._rain_map = fr

    def add_river(self, xstart: float, xend: float, ystart: float, yend: float, times, q) -> float:
        """A river discharging q(t) (m^3/s) over the cells its box overlaps; returns
        the discharge area (0: the box misses every cell and the river is dropped)."""
        t = np.ascontiguousarray(times, np.float64)
        qq = np.ascontiguousarray(q, np.float64)
        a = ctypes.c_double(0.0)
        _check(lib().bgf_add_river(self.handle, float(xstart), float(xend), float(ystart), float(yend), len(t),
                                   t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   qq.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(a)),
               "bgf_add_river")
        return a.value

    def set_state(self, h: np.ndarray, u: np.ndarray, v: np.ndarray) -> None:
        hh, uu, vv = (np.ascontiguousarray(a, self.dtype) for a in (h, u, v))
        ev = CEvolving(None, _ptr(hh), _ptr(uu), _ptr(vv))
        _check(lib().bgf_set_state(self.handle, ctypes.byref(ev)), "bgf_set_state")

    def get_state(self, out=None):
        """Returns (zs, h, u, v) as (nblkmem, 18, 18) arrays (interior cells filled).
        ``out``: four such arrays of the handle's field type to fill instead of new ones."""
        if out is None:
            out = [np.zeros((self.nblkmem, 18, 18), self.dtype) for _ in range(4)]
        else:
            out = list(out)
            for a in out:
                if a.dtype != self.dtype or a.shape != (self.nblkmem, 18, 18) or not a.flags.c_contiguous:
                    raise ValueError("get_state: out arrays must be C-contiguous (nblkmem, 18, 18) of the field type")
        ev = CEvolving(*[_ptr(a) for a in out])
        _check(lib().bgf_get_state(self.handle, ctypes.byref(ev)), "bgf_get_state")
        return tuple(out)

    def set_grid(self, grid: int) -> None:
        """CTAs of the fused kernels (0: one per block; fewer: persistent launch)."""
        _check(lib().bgf_set_grid(self.handle, int(grid)), "bgf_set_grid")

    def set_gauges(self, gauges) -> None:
        """Gauge cells (block id, i, j) sampled after every step (the reference's
        time-series output nodes)."""
        g = np.asarray(list(gauges), np.int32).reshape(-1, 3)
        cols = [np.ascontiguousarray(g[:, k]) for k in range(3)]
        _check(lib().bgf_set_gauges(self.handle, len(g), *[_ptr(c) for c in cols]), "bgf_set_gauges")
        self._ngauges = len(g)

    def read_gauges(self, max_samples: int = 1 << 20):
        """(times (s, n), values (s, n, 4) as h, zs, u, v, lost) of the samples
        recorded since the last read."""
        n = max(getattr(self, "_ngauges", 0), 1)
        t = np.zeros((max_samples, n))
        v = np.zeros((max_samples, n, 4))
        ns = ctypes.c_int(0)
        lost = ctypes.c_int64(0)
        _check(lib().bgf_read_gauges(self.handle, int(max_samples), _ptr(t), _ptr(v), ctypes.byref(ns),
                                     ctypes.byref(lost)), "bgf_read_gauges")
        return t[:ns.value], v[:ns.value], lost.value

    def set_kernel_layout(self, cells_per_thread: int) -> None:
        """Thread layout of the fused single-level kernels: 2 cells per thread (default),
        1, or 3 (two cells per thread in persistent CTAs with a staging warp)."""
        _check(lib().bgf_set_kernel_layout(self.handle, int(cells_per_thread)), "bgf_set_kernel_layout")

    def autotune(self, loop: Loop, steps: int = 20) -> tuple:
        """Times the step kernels for each launch shape from the state of ``loop`` and
        keeps the fastest; the state is unchanged afterwards.  Returns (grid, ms_per_step)."""
        c = loop.to_c()
        g = ctypes.c_int(0)
        ms = ctypes.c_double(0.0)
        _check(lib().bgf_autotune(self.handle, ctypes.byref(c), int(steps), ctypes.byref(g), ctypes.byref(ms)),
               "bgf_autotune")
        return g.value, ms.value

    def get_bed(self) -> np.ndarray:
        """zb on (nblkmem, 18, 18) tiles, halo included."""
        out = np.zeros((self.nblkmem, 18, 18), self.dev_dtype)
        _check(lib().bgf_get_bed(self.handle, _ptr(out)), "bgf_get_bed")
        return out

    # -- refinement pass ---------------------------------------------------------------
    def set_bathy(self, xo: float, yo: float, dx: float, grid: np.ndarray) -> None:
        """Bathymetry grid (ny, nx) of nodes from (xo, yo) with spacing dx."""
        g = np.ascontiguousarray(grid, np.float32)
        ny, nx = g.shape
        _check(lib().bgf_set_bathy(self.handle, nx, ny, float(xo), float(yo), float(dx), _ptr(g)), "bgf_set_bathy")

    def add_target_level_map(self, xo: float, yo: float, dx: float, levels: np.ndarray) -> None:
        """Target-level map (ny, nx) of integer levels, node (0, 0) at (xo, yo), for the
        Targetlevel criterion; maps apply in the order added (the last decides)."""
        g = np.ascontiguousarray(levels, np.int32)
        ny, nx = g.shape
        _check(lib().bgf_add_target_level_map(self.handle, nx, ny, float(xo), float(yo), float(dx),
                                              g.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
               "bgf_add_target_level_map")

    def clear_target_level_maps(self) -> None:
        _check(lib().bgf_clear_target_level_maps(self.handle), "bgf_clear_target_level_maps")

    def _adapt_param(self, crit, maxiteration: int, allow_coarsen: bool = False):
        from .adapt import VARS
        return CAdaptParam(crit.kind, VARS[crit.var], float(crit.arg1), float(crit.arg2), int(maxiteration),
                           1 if allow_coarsen else 0)

    def adapt_flags(self, crit, allow_coarsen: bool = False):
        """(refine, coarsen) per active block of one criterion + sanity pass; with
        allow_coarsen, coarsen marks the parents of the quads that would merge."""
        n = ctypes.c_int(0)
        _check(lib().bgf_get_blocks(self.handle, ctypes.byref(n), None, None, None, None, None), "bgf_get_blocks")
        r = np.zeros(n.value, np.uint8)
        c = np.zeros(n.value, np.uint8)
        p = self._adapt_param(crit, 1, allow_coarsen)
        _check(lib().bgf_adapt_flags(self.handle, ctypes.byref(p), _ptr(r), _ptr(c)), "bgf_adapt_flags")
        return r, c

    def adapt(self, crit, maxiteration: int = 20, allow_coarsen: bool = False):
        """Adaptation of the mesh and state; returns (nblk, passes).  allow_coarsen
        (an extension; the reference cancels coarsening) also merges quads."""
        p = self._adapt_param(crit, maxiteration, allow_coarsen)
        n, it = ctypes.c_int(0), ctypes.c_int(0)
        _check(lib().bgf_adapt(self.handle, ctypes.byref(p), ctypes.byref(n), ctypes.byref(it)), "bgf_adapt")
        return n.value, it.value

    def set_adapt_mode(self, mode: int) -> None:
        """1 (default): adaptation tables on the device when the mesh allows; 0: host tables."""
        _check(lib().bgf_set_adapt_mode(self.handle, int(mode)), "bgf_set_adapt_mode")

    def get_blocks(self):
        """(active, level, nbr (nblkmem, 8), xo, yo) host copies of the tables."""
        n = ctypes.c_int(0)
        act = np.zeros(self.nblkmem, np.int32)
        lev = np.zeros(self.nblkmem, np.int32)
        nb = np.zeros((self.nblkmem, 8), np.int32)
        xo = np.zeros(self.nblkmem)
        yo = np.zeros(self.nblkmem)
        _check(lib().bgf_get_blocks(self.handle, ctypes.byref(n), _ptr(act), _ptr(lev), _ptr(nb), _ptr(xo), _ptr(yo)),
               "bgf_get_blocks")
        return act[: n.value], lev, nb, xo, yo

    # -- time stepping --------------------------------------------------------------
    def init_dt(self, loop: Loop) -> float:
        c = loop.to_c()
        _check(lib().bgf_init_dt(self.handle, ctypes.byref(c)), "bgf_init_dt")
        loop.from_c(c)
        return loop.dtmax

    def flow_step(self, loop: Loop) -> float:
        """One step (FlowGPU equivalent); returns dt and leaves totaltime to the caller."""
        c = loop.to_c()
        _check(lib().bgf_flow_step(self.handle, ctypes.byref(c)), "bgf_flow_step")
        loop.from_c(c)
        return loop.dt

    def run(self, loop: Loop, endtime: float, outputtimestep: float = 0.0, maxsteps: int = 2**31 - 1) -> int:
        c = loop.to_c()
        n = ctypes.c_int(0)
        rc = lib().bgf_run(self.handle, ctypes.byref(c), float(endtime), float(outputtimestep), int(maxsteps),
                           ctypes.byref(n))
        loop.from_c(c)
        _check(rc, "bgf_run")
        return n.value

    def volume(self) -> float:
        v = ctypes.c_double(0.0)
        _check(lib().bgf_volume(self.handle, ctypes.byref(v)), "bgf_volume")
        return v.value

    def kernel_launches(self) -> int:
        return int(lib().bgf_kernel_launches(self.handle))

    def set_profiling(self, on: bool) -> None:
        _check(lib().bgf_set_profiling(self.handle, 1 if on else 0), "bgf_set_profiling")

    def kernel_timing(self):
        """(flux_ms, update_ms, steps) accumulated by bgf_flow_step while profiling is on."""
        a, b = ctypes.c_double(0), ctypes.c_double(0)
        n = ctypes.c_int64(0)
        _check(lib().bgf_kernel_timing(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n)),
               "bgf_kernel_timing")
        return a.value, b.value, n.value

    def last_run_timing(self):
        """(gpu_ms, kernel launches) of the last run()."""
        ms = ctypes.c_double(0)
        n = ctypes.c_int64(0)
        _check(lib().bgf_run_timing(self.handle, ctypes.byref(ms), ctypes.byref(n)), "bgf_run_timing")
        return ms.value, n.value


def build_model(param: Param, zb: np.ndarray, h: np.ndarray, u: np.ndarray | None = None, v: np.ndarray | None = None,
                cf: np.ndarray | None = None, rain: tuple | None = None, mesh: Mesh | None = None) -> tuple:
    """Builds a FlowB200 scenario from row-major (ny, nx) cell arrays on a uniform
    level-0 mesh: block tables, bed with filled halo, boundary segments (declared
    segments plus the remainder of type ``aoibnd``), optional per-cell cf and a
    uniform rain series (times, mm/h).  Returns (FlowB200, Mesh)."""
    ny, nx = zb.shape
    mesh = mesh or uniform_mesh(nx, ny, param.dx, doubleprecision=bool(param.doubleprecision))
    dt = np.float64 if (param.doubleprecision or param.splitprecision) else np.float32
    f = FlowB200(param, mesh.nblk)
    f.set_blocks(mesh.active, mesh.level, mesh.nbr, mesh.xo, mesh.yo)
    zbb = fill_halo(grid_to_buq(np.asarray(zb, np.float64).astype(dt).astype(np.float64), mesh), mesh)
    cfb = None if cf is None else grid_to_buq(np.asarray(cf, np.float64), mesh)
    act = _rain_mask(zbb, param.mask) if rain is not None else None
    f.set_bed(zbb, cf=cfb, activeCell=act)
    xo = 0.0 if math.isnan(param.xo) else param.xo
    yo = 0.0 if math.isnan(param.yo) else param.yo
    for typ, times, levels, sides in boundary_segments(mesh, param.segments, param.aoibnd, xo, yo):
        f.add_segment(typ, times, levels, sides)
    if rain is not None:
        f.set_rain(rain[0], rain[1])
    u = np.zeros_like(h) if u is None else u
    v = np.zeros_like(h) if v is None else v
    f.set_state(grid_to_buq(h, mesh), grid_to_buq(u, mesh), grid_to_buq(v, mesh))
    return f, mesh


def _rain_mask(zbb: np.ndarray, mask: float) -> np.ndarray | None:
    """activeCell as calcactiveCellCPU leaves it (src/InitialConditions.cu:1560-1610):
    1 where zb < mask.  Its boundary-row exclusion for rainbnd = false loops over the
    legacy side lists, whose counts stay 0 because the calls that fill them are
    commented out (src/InitialConditions.cu:77-78), so it removes nothing.
    Returns None when every cell is active."""
    act = (np.asarray(zbb) < mask).astype(np.int32)
    return None if act.all() else act
