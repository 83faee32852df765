"""Synthetic test cases shared by the tests, smoke() and bench.py.

Every case is a regular grid of nx*ny cells (multiples of 16) with bed zb and an
initial state, plus the parameters, boundary segments and forcing series of a
BG_Flood run.  Fields are generated in float32 so that the reference, the
oracle and the GPU library all start from identical values.  The shapes and
value ranges follow the synthetic workloads of the flow-step benchmark
(Gaussian hump, conical island with a solitary wave, rain on fractal terrain);
all are generated from fixed seeds, none is read from a data set.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from bg_flood_b200.params import BndSegmentSpec, Param


@dataclass
class Case:
    name: str
    param: Param
    paramtext: str          # the same parameters as reference BG_param.txt lines
    dx: float
    xo: float
    yo: float
    zb: np.ndarray          # (ny, nx) float32
    h: np.ndarray
    u: np.ndarray
    v: np.ndarray
    cf: np.ndarray | None = None
    rain: tuple | None = None  # (times, mm/h)
    nextoutputtime: float = 1e30

    @property
    def nx(self):
        return self.zb.shape[1]

    @property
    def ny(self):
        return self.zb.shape[0]


def _cell_centres(nx, ny, dx, xo, yo):
    x = (xo + (np.arange(nx) + 0.5) * dx).astype(np.float64)
    y = (yo + (np.arange(ny) + 0.5) * dx).astype(np.float64)
    return np.meshgrid(x, y)


def _param_text(p: Param, extra: str = "") -> str:
    lines = [f"CFL = {p.CFL!r}", f"theta = {p.theta!r}", f"eps = {p.eps!r}", f"cf = {p.cf!r}",
             f"frictionmodel = {p.frictionmodel}", f"aoibnd = {p.aoibnd}", "gpudevice = -1",
             f"harness_engine = {p.engine}"]
    if not math.isnan(p.zsinit):
        lines.append(f"zsinit = {p.zsinit!r}")
    if p.ForceMassConserve:
        lines.append("ForceMassConserve = 1")
    for s in p.segments:
        lines.append(f"{s.side} = {s.type}")
    return "\n".join(lines) + "\n" + extra


def gauss(n: int = 64, engine: int = 1, aoibnd: int = 3) -> Case:
    """The reference's Gaussian-hump set-up (src/Testing.cu:418-551) on an n*n grid:
    dx = 1/256, still water at 0.1 over a flat bed at 0 plus a hump of amplitude 1
    and radius 0.05, absorbing remainder boundary by default."""
    dx = 1.0 / 256
    xo = yo = -n / 512.0
    X, Y = _cell_centres(n, n, dx, xo, yo)
    f32 = np.float32
    zs = (f32(0.1) + np.exp(-(X * X + Y * Y) / (2 * 0.05 ** 2))).astype(f32)
    p = Param(dx=dx, xo=xo, yo=yo, engine=engine, aoibnd=aoibnd, zsinit=0.1, cf=0.0, frictionmodel=0)
    z = np.zeros((n, n), f32)
    return Case(f"gauss{n}_e{engine}_b{aoibnd}", p, _param_text(p), dx, xo, yo, z, zs.copy(), z.copy(), z.copy(),
                nextoutputtime=0.1)


def hump_walls(n: int = 256, engine: int = 2) -> Case:
    """Plain single-level case: n*n cells, dx = 1 m, flat bed at -1 m, eta = 0.1
    exp(-r^2 / (2 * 20^2)) centred, u = v = 0, reflective walls, no friction."""
    dx = 1.0
    xo = yo = 0.0
    X, Y = _cell_centres(n, n, dx, xo, yo)
    c = n * dx / 2
    r2 = (X - c) ** 2 + (Y - c) ** 2
    eta = (0.1 * np.exp(-r2 / (2 * 20.0 ** 2))).astype(np.float32)
    zb = np.full((n, n), -1.0, np.float32)
    h = (eta - zb).astype(np.float32)
    p = Param(dx=dx, xo=xo, yo=yo, engine=engine, aoibnd=0, cf=0.0, frictionmodel=0)
    z = np.zeros((n, n), np.float32)
    return Case(f"hump{n}_e{engine}", p, _param_text(p), dx, xo, yo, zb, h, z, z.copy())


def conical_island(n: int = 128, engine: int = 1, dx: float | None = None, wave: bool = True) -> Case:
    """Wet/dry run-up: flat bed 0.32 m deep with a conical island (base radius 3.6 m,
    top radius 1.1 m, crest 0.625 m above the bed) at the centre, Manning n = 0.01,
    and a solitary wave (A = 0.032 m, sech^2 profile) imposed as a Dirichlet water
    level on the west side.  n = 1024 with dx = 0.05 m is the full-size workload."""
    dx = dx if dx is not None else 25.6 / n
    xo = yo = 0.0
    X, Y = _cell_centres(n, n, dx, xo, yo)
    c = n * dx / 2
    r = np.sqrt((X - c) ** 2 + (Y - c) ** 2)
    cone = np.clip((3.6 - r) / (3.6 - 1.1), 0.0, 1.0) * 0.625
    zb = (-0.32 + cone).astype(np.float32)
    h = np.maximum(0.0 - zb, 0.0).astype(np.float32)
    p = Param(dx=dx, xo=xo, yo=yo, engine=engine, aoibnd=0, cf=0.01, frictionmodel=-1)
    if wave:
        A, depth = 0.032, 0.32
        k = math.sqrt(3 * A / (4 * depth ** 3))
        cel = math.sqrt(9.81 * depth * (1 + A / depth))
        t = np.linspace(0.0, 20.0, 201)
        x0 = 2.5 / k
        wl = A / np.cosh(k * (cel * t - x0)) ** 2
        p.segments = [BndSegmentSpec("left", 2, list(t), list(wl))]
    z = np.zeros((n, n), np.float32)
    return Case(f"island{n}_e{engine}", p, _param_text(p), dx, xo, yo, zb, h, z, z.copy())


def fractal_terrain(n: int, seed: int, relief: float = 300.0, slope: float = -2.0) -> np.ndarray:
    """Seeded spectral synthesis: power spectrum ~ k^slope, rescaled to 0..relief,
    with a carved valley along the middle row."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(n)[None, :]
    ky = np.fft.fftfreq(n)[:, None]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = 1.0
    amp = k ** (slope / 2.0)
    amp[0, 0] = 0.0
    phase = rng.uniform(0, 2 * np.pi, (n, n))
    z = np.real(np.fft.ifft2(amp * np.exp(1j * phase)))
    z = (z - z.min()) / (z.max() - z.min()) * relief
    yy = np.arange(n)[:, None] / n
    valley = np.exp(-((yy - 0.5) / 0.08) ** 2)
    return (z * (1 - 0.8 * valley)).astype(np.float32)


def rain_on_terrain(n: int = 64, engine: int = 1, dx: float = 10.0, seed: int = 7, rain_mmh: float = 50.0,
                    manning: float = 0.035) -> Case:
    """Rain on grid: seeded fractal terrain (0-300 m relief), dry start, uniform rain
    for one hour, Manning friction, walls."""
    zb = fractal_terrain(n, seed)
    h = np.zeros((n, n), np.float32)
    p = Param(dx=dx, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=manning, frictionmodel=-1)
    z = np.zeros((n, n), np.float32)
    rain = ([0.0, 3600.0, 3601.0, 1e9], [rain_mmh, rain_mmh, 0.0, 0.0])
    return Case(f"rain{n}_e{engine}", p, _param_text(p), dx, 0.0, 0.0, zb, h, z, z.copy(), rain=rain)


def dam_break(n: int = 64, engine: int = 1, seed: int = 3) -> Case:
    """Wet/dry: a 1 m step of water over a sloping, noisy bed with a dry downstream
    part, quadratic friction, walls, random initial velocities."""
    rng = np.random.default_rng(seed)
    dx = 0.5
    X, Y = _cell_centres(n, n, dx, 0.0, 0.0)
    zb = (0.02 * X + 0.05 * rng.standard_normal((n, n))).astype(np.float32)
    eta = np.where(X < n * dx / 3, 1.2, 0.0)
    h = np.maximum(eta - zb, 0.0).astype(np.float32)
    u = np.where(h > 0, 0.2 * rng.standard_normal((n, n)), 0.0).astype(np.float32)
    v = np.where(h > 0, 0.2 * rng.standard_normal((n, n)), 0.0).astype(np.float32)
    p = Param(dx=dx, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=0.002, frictionmodel=0)
    return Case(f"dam{n}_e{engine}", p, _param_text(p), dx, 0.0, 0.0, zb, h, u, v)


# ---------------------------------------------------------------- multi-level meshes

@dataclass
class AMRCase:
    """A case on a mesh refined by the reference's own Adaptation(): fields are
    functions of cell-centre coordinates, sampled on the level-0 grid before the
    adaptation and again on every block of the adapted mesh."""
    name: str
    param: Param
    paramtext: str
    n0: int                 # level-0 cells per side
    dx: float               # level-0 resolution
    xo: float
    yo: float
    zb_fn: object
    eta_fn: object
    uv_fn: object = None
    nextoutputtime: float = 1e30
    adapt_eta_fn: object = None   # surface used only to drive the adaptation (default eta_fn)


def _amr_text(p: Param, crit: str, maxlevel: int) -> str:
    p.initlevel, p.minlevel, p.maxlevel = 0, 0, maxlevel
    return _param_text(p) + f"initlevel = 0\nminlevel = 0\nmaxlevel = {maxlevel}\nAdaptation = {crit}\n"


def amr_hump(n0: int = 32, engine: int = 1, maxlevel: int = 1, off: float = 0.5) -> AMRCase:
    """Gaussian hump on a flat bed, refined where the surface exceeds 0.13 m; the hump
    sits at fraction `off` of the domain (off-centre gives a mixed-level mesh)."""
    dx = 1.0 / 64
    p = Param(dx=dx, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=0.0, frictionmodel=0)
    c = n0 * dx * off
    eta = lambda x, y: 0.1 + 0.5 * np.exp(-((x - c) ** 2 + (y - c) ** 2) / (2 * 0.05 ** 2))
    return AMRCase(f"amrhump{n0}_e{engine}_l{maxlevel}", p, _amr_text(p, "Threshold,0.13,zs", maxlevel), n0, dx, 0.0,
                   0.0, lambda x, y: np.zeros_like(x), eta)


def amr_island(n0: int = 32, engine: int = 1, maxlevel: int = 2, off: float = 0.5) -> AMRCase:
    """Conical island with a wet/dry shoreline, refined on the island (bed above
    -0.2 m), quadratic friction, a small tilted surface to drive a flow."""
    dx = 0.4
    p = Param(dx=dx, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=0.001, frictionmodel=0)
    c = n0 * dx * off

    def zb(x, y):
        r = np.sqrt((x - c) ** 2 + (y - c) ** 2)
        return -0.32 + np.clip((3.6 - r) / 2.5, 0.0, 1.0) * 0.625

    eta = lambda x, y: 0.01 * (x - c) / c
    return AMRCase(f"amrisland{n0}_e{engine}_l{maxlevel}", p, _amr_text(p, "Threshold,-0.2,zb", maxlevel), n0, dx,
                   0.0, 0.0, zb, eta)


def amr_dambreak(n0: int = 64, engine: int = 1, maxlevel: int = 2, seed: int = 5) -> AMRCase:
    """Wet/dry on a three-level mesh: a noisy sloping bed, water up to 1.2 m left of
    x = 0.45 L and dry land beyond; the mesh is refined around the left third, so the
    wet/dry front crosses level interfaces."""
    dx = 0.5
    L = n0 * dx
    p = Param(dx=dx, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=0.002, frictionmodel=0)
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(64)

    def zb(x, y):
        return 0.02 * x + 0.05 * np.sin(x * 1.3 + noise[0]) * np.cos(y * 0.7 + noise[1])

    eta = lambda x, y: np.where(x < 0.45 * L, 1.2, -10.0)
    crit = lambda x, y: np.where(x < 0.33 * L, 2.0, -10.0)
    return AMRCase(f"amrdam{n0}_e{engine}_l{maxlevel}", p, _amr_text(p, "Threshold,0.5,zs", maxlevel), n0, dx, 0.0,
                   0.0, zb, eta, adapt_eta_fn=crit)


# ---------------------------------------------------------------- ensembles

def _blocks_grid(nblocks: int, rng) -> tuple[int, int]:
    """Block columns and rows of a near-square grid with about nblocks blocks."""
    nbx = max(1, int(round(math.sqrt(nblocks) * rng.uniform(0.8, 1.25))))
    nby = max(1, int(round(nblocks / nbx)))
    return nbx, nby


def ensemble_member(k: int, seed: int, min_blocks: int = 64, max_blocks: int = 16384, engine: int = 1) -> Case:
    """Member k of a seeded ensemble: block count log-uniform in [min_blocks,
    max_blocks]; three in four members are rain on fractal terrain (0-300 m relief,
    rain 10-100 mm/h, Manning n in [0.02, 0.06], dx = 10 m), one in four a tsunami
    (bed -4000..-200 m with a seamount ridge, initial Gaussian surface hump of
    0.01-1 m, dx = 500 m, no friction).  Walls on all sides."""
    rng = np.random.default_rng([seed, k])
    nblocks = int(round(math.exp(rng.uniform(math.log(min_blocks), math.log(max_blocks)))))
    nbx, nby = _blocks_grid(nblocks, rng)
    nx, ny = 16 * nbx, 16 * nby
    z = np.zeros((ny, nx), np.float32)
    if k % 4 != 3:
        m = max(nx, ny)
        zb = fractal_terrain(m, int(rng.integers(1 << 30)))[:ny, :nx].copy()
        rain_mmh = float(rng.uniform(10.0, 100.0))
        manning = float(rng.uniform(0.02, 0.06))
        p = Param(dx=10.0, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=manning, frictionmodel=-1)
        rain = ([0.0, 3600.0, 3601.0, 1e9], [rain_mmh, rain_mmh, 0.0, 0.0])
        return Case(f"ens{seed}_{k}_rain_{nbx}x{nby}", p, _param_text(p), 10.0, 0.0, 0.0, zb,
                    np.zeros((ny, nx), np.float32), z, z.copy(), rain=rain)
    dx = 500.0
    X, Y = _cell_centres(nx, ny, dx, 0.0, 0.0)
    L = nx * dx
    zb = (-4000.0 + 3800.0 * np.exp(-((X - 0.7 * L) / (0.08 * L)) ** 2)).astype(np.float32)
    amp = float(rng.uniform(0.01, 1.0))
    eta = amp * np.exp(-((X - 0.3 * L) ** 2 + (Y - 0.5 * ny * dx) ** 2) / (2 * (0.05 * L) ** 2))
    h = np.maximum(eta - zb, 0.0).astype(np.float32)
    p = Param(dx=dx, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=0.0, frictionmodel=0)
    return Case(f"ens{seed}_{k}_tsunami_{nbx}x{nby}", p, _param_text(p), dx, 0.0, 0.0, zb, h, z, z.copy())
