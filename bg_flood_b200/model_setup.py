"""A scenario from its ``BG_param.txt``: the reference's start-up, host side.

``prepare_model`` follows the reference's ``main`` up to the time loop
(src/BG_Flood.cu:55-156) for the inputs this library covers:

1. Readparamfile (src/ReadInput.cu:57-95): keys and aliases of params.py, the
   bathymetry, rain and boundary file keys;
2. readforcing (src/ReadForcing.cu:38-53, 75-97, 250-280, 365-381): bathymetry
   grid, uniform boundary series, river discharge series (the run's end and start
   times are fitted into each river's time range), uniform rain series;
3. checkparamsanity (src/ReadInput.cu:1189-1480): level defaults, rain forces
   double precision, zsoffset, domain extent from the bathymetry, nx/ny rounded
   up to whole blocks, end time and output times;
4. InitMesh (src/Mesh.cu:36-160, 257-433): blocks whose cells all lie above
   ``mask`` are dropped, tables in the reference's order;
5. InitialConditions (src/InitialConditions.cu:23-120): bed by interp2BUQ and
   setedges, cold start (zs = max(zsinit + zsoffset, zb)) or, with no zsinit and
   a boundary series, the warm start from the series' mean level
   (src/InitEvolv.cu:36-290), rivers (discharge areas, InitRivers), boundary
   blocks, rain mask;
6. InitialAdaptation (src/Adaptation.cu:133-146) when maxlevel != minlevel: the
   refinement pass on the device, then step 5 again on the refined mesh;
7. InitLoop and the first map output (src/Mainloop.cu:207-240, 323-340).

``setup_model`` then loads the result into a FlowB200 handle and returns it
with its Loop, ready for ``run``.

Inputs outside this library's scope raise ValueError: netCDF or other grid
formats, several bathymetry layers, roughness / infiltration / deformation
maps, wind, atmospheric pressure, AOI polygons, spherical grids, engine 5,
hot starts.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np

from ._native import lib
from .mesh import Mesh, boundary_segments, uniform_mesh
from .params import Param, read_param_text
from .readforcing import BathyGrid, read_asc, read_bathy, read_flow_file, read_uniform_series

__all__ = ["ModelInputs", "read_param_file", "prepare_model", "setup_model", "check_param_sanity", "inputs_on_mesh"]

_TINY = 0.0000001
_DEFAULT_ENDTIME = Param().endtime


@dataclass
class ModelInputs:
    """Host arrays of a set-up scenario, BUQ tiles (nblk, 18, 18) in block order."""
    param: Param
    bathy: BathyGrid
    mesh: Mesh
    zb: np.ndarray          # interior from interp2BUQ + setedges, halo 0 (filled on the device)
    h: np.ndarray
    u: np.ndarray
    v: np.ndarray
    zs: np.ndarray          # the reference's initial surface (the device keeps zs = zb + h)
    active_cell: np.ndarray | None
    segments: list          # (type, times, levels, [left, right, top, bot] blocks)
    rain: tuple | None      # (times s, mm/h)
    rivers: list            # (xstart, xend, ystart, yend, times, discharges m^3/s)
    output_times: list
    totaltime: float
    nextoutputtime: float
    nblkmem: int
    adapted: bool = False
    notes: list = field(default_factory=list)


def _resolve(path: str, basedir: str) -> str:
    return path if os.path.isabs(path) else os.path.join(basedir, path)


def read_param_file(path: str) -> Param:
    """Readparamfile: every line of the file through the key reader (lines starting
    with ``#`` skipped).  Unsupported input keys raise."""
    with open(path, "r") as fh:
        text = fh.read()
    lines = [ln for ln in text.splitlines() if ln and not ln.startswith("#")]
    _reject_unsupported(lines)
    p = read_param_text("\n".join(lines))
    if p.cf_file:
        raise ValueError(f"roughness map '{p.cf_file}' (cf key) is not supported by this library")
    return p


# keys of inputs this library does not read (readparamstr, src/ReadInput.cu:890-1180)
_UNSUPPORTED = {
    "aoi": "AOI polygons", "aoipoly": "AOI polygons", "cfmap": "roughness maps",
    "roughnessmap": "roughness maps", "wind": "wind forcing", "windfiles": "wind forcing", "atmp": "pressure forcing",
    "atmpfile": "pressure forcing", "deform": "deformation", "hotstartfile": "hot start", "hotstart": "hot start",
    "initiallossmap": "infiltration maps", "ilmap": "infiltration maps", "continuouslossmap": "infiltration maps",
    "clmap": "infiltration maps", "spherical": "spherical grids",
}


def _reject_unsupported(lines: list) -> None:
    for ln in lines:
        body = ln.split("#", 1)[0]
        if "=" not in body:
            continue
        key, val = body.split("=", 1)
        k = key.strip().lower()
        v = val.split(";", 1)[0].strip()
        if k in _UNSUPPORTED and v and not (k == "spherical" and v in ("0", "false", "no")):
            raise ValueError(f"BG_param key '{key.strip()}' ({_UNSUPPORTED[k]}) is not supported by this library")


def _ftoi(v: float) -> int:
    # ftoi (src/Util_CPU.cu:308-311): round half away from zero
    return int(v + 0.5) if v >= 0 else int(v - 0.5)


def _calcres(dx: float, level: int) -> float:
    return dx * (1 << -level) if level < 0 else dx / (1 << level)


def check_param_sanity(p: Param, bathy: BathyGrid, rain_file: bool) -> list:
    """checkparamsanity for the covered keys; mutates p, returns the output times."""
    minlev = p.initlevel if p.minlevel == -99999 else p.minlevel
    maxlev = p.initlevel if p.maxlevel == -99999 else p.maxlevel
    p.maxlevel = max(maxlev, minlev)
    p.minlevel = min(maxlev, minlev)
    p.initlevel = min(max(p.minlevel, p.initlevel), p.maxlevel)
    if rain_file:
        p.doubleprecision = 1  # the reference forces double for rain-on-grid cases
    p.zsoffset = 0.0 if math.isnan(p.zsoffset) else p.zsoffset
    if math.isnan(p.xo):
        p.xo = bathy.xo - 0.5 * bathy.dx
    if math.isnan(p.xmax):
        p.xmax = bathy.xmax + 0.5 * bathy.dx
    if math.isnan(p.yo):
        p.yo = bathy.yo - 0.5 * bathy.dx
    if math.isnan(p.ymax):
        p.ymax = bathy.ymax + 0.5 * bathy.dx
    if math.isnan(p.dx):
        p.dx = bathy.dx
    if math.isnan(p.grdalpha):
        p.grdalpha = bathy.grdalpha
    levdx = _calcres(p.dx, p.initlevel)
    nx = _ftoi((p.xmax - p.xo) / levdx) or 1
    ny = _ftoi((p.ymax - p.yo) / levdx) or 1
    p.xmax = p.xo + (math.ceil(nx / 16.0) * 16.0) * levdx
    p.ymax = p.yo + (math.ceil(ny / 16.0) * 16.0) * levdx
    p.grdalpha = p.grdalpha * math.pi / 180.0
    if p.engine == 5:
        raise ValueError("engine 5 (multi-layer) is not supported by this library")
    if abs(p.endtime - _DEFAULT_ENDTIME) <= _TINY:
        p.endtime = 1.0 / _TINY
    p.inittime = p.totaltime
    # Toutput from outputtimestep (src/ReadInput.cu:1445-1475), sorted and unique
    if abs(p.outputtimestep - Param().outputtimestep) <= _TINY:
        times = [p.totaltime, p.endtime]
    else:
        nstep = int((p.endtime - p.totaltime) / p.outputtimestep + 1)
        times = [min(p.totaltime + p.outputtimestep * k, p.endtime) for k in range(nstep)] + [p.endtime]
    times = [min(max(p.totaltime, t), p.endtime) for t in times if t >= p.totaltime] or [p.totaltime]
    return sorted(set(times))


def _model_dtype(p: Param):
    return np.float64 if p.doubleprecision else np.float32


def _mesh_counts(p: Param) -> tuple:
    levdx = _calcres(p.dx, p.initlevel)
    nx = _ftoi((p.xmax - p.xo) / levdx)
    ny = _ftoi((p.ymax - p.yo) / levdx)
    return nx, ny, levdx


def _interp_bed(bathy: BathyGrid, p: Param, nblk: int, level, nbr, bxo, byo) -> np.ndarray:
    zb = np.zeros((nblk, 18, 18), np.float64)
    g = bathy.to_c()
    lv = np.ascontiguousarray(level[:nblk], np.int32)
    nb = np.ascontiguousarray(nbr[:nblk], np.int32)
    xo = np.ascontiguousarray(bxo[:nblk], np.float64)
    yo = np.ascontiguousarray(byo[:nblk], np.float64)
    rc = lib().bgf_interp_bathy(ctypes.byref(g), nblk, lv.ctypes.data, nb.ctypes.data, xo.ctypes.data,
                                yo.ctypes.data, float(p.xo), float(p.yo), float(p.dx), int(bool(p.doubleprecision)),
                                zb.ctypes.data)
    if rc != 0:
        raise ValueError(f"bgf_interp_bathy: {lib().bgf_last_error().decode()}")
    return zb


def _initial_state(p: Param, zb: np.ndarray, segments: list) -> tuple:
    """initevolv: cold start, or the warm start from uniform boundary series."""
    T = _model_dtype(p)
    zbT = zb.astype(T)
    bndison = any(s.file for s in p.segments)
    zsinit = p.zsinit
    if math.isnan(zsinit) and not bndison:
        zsinit = 0.0
    if not math.isnan(zsinit):
        zz = T(zsinit) + T(p.zsoffset)
    else:
        # warmstart (src/InitEvolv.cu:180-290): mean over the uniform series of the
        # level interpolated at totaltime, first sample pair whose end is >= totaltime
        acc, nuni = T(0.0), 0
        for s in p.segments:
            if not s.file:
                continue
            t, w = np.asarray(s.times, np.float64), np.asarray(s.levels, np.float64)
            k = 1
            while k < len(t) and t[k] - p.totaltime < 0.0:
                k += 1
            if k >= len(t):
                raise ValueError(f"boundary series {s.file} ends before the start time")
            val = w[k - 1] + (p.totaltime - t[k - 1]) / (t[k] - t[k - 1]) * (w[k] - w[k - 1])
            acc = T(float(acc) + val)  # T accumulator plus a double sample, rounded to T
            nuni += 1
        zz = T(acc / T(nuni))
    zs = np.zeros_like(zbT)
    h = np.zeros_like(zbT)
    inner = (slice(None), slice(1, 17), slice(1, 17))
    zs[inner] = np.where(zz > zbT[inner], zz, zbT[inner])
    d = (zs[inner] - zbT[inner]).astype(T)
    h[inner] = np.where(d > T(0.0), d, T(0.0))
    return zs.astype(np.float64), h.astype(np.float64)


def _boundary_series(p: Param, basedir: str, reftime: list) -> None:
    for s in p.segments:
        if s.file:
            path = _resolve(s.file, basedir)
            if path.lower().endswith(".nc") or "?" in os.path.basename(path):
                raise ValueError(f"gridded boundary forcing is not supported by this library: {s.file}")
            t, w = read_uniform_series(path, reftime)
            s.times, s.levels = list(t), list(w)


def _river_series(p: Param, basedir: str, reftime: list) -> list:
    """readforcing's river part: the discharge series, and the end and start times
    fitted into each river's time range."""
    out = []
    for fname, xs, xe, ys, ye in p.rivers:
        t, q = read_flow_file(_resolve(fname, basedir), reftime)
        if t[-1] < p.endtime:
            p.endtime = float(t[-1])
        if t[0] > p.totaltime:
            p.totaltime = float(t[0])
        out.append((xs, xe, ys, ye, t, q))
    return out


def _rain_series(p: Param, basedir: str, reftime: list):
    if not p.rain:
        return None
    path = _resolve(p.rain, basedir)
    if path.lower().endswith(".nc") or "?" in os.path.basename(path):
        raise ValueError(f"gridded rain forcing is not supported by this library: {p.rain}")
    return read_uniform_series(path, reftime)


def _initial_conditions(p: Param, bathy: BathyGrid, mesh: Mesh, level, nbr, bxo, byo) -> dict:
    nblk = mesh.nblk
    zb = _interp_bed(bathy, p, nblk, level, nbr, bxo, byo)
    zs, h = _initial_state(p, zb, p.segments)
    segs = boundary_segments(mesh, p.segments, p.aoibnd, p.xo, p.yo)
    # calcactiveCellCPU (src/InitialConditions.cu:1560-1610): 1 where zb < mask; only
    # the rain source reads it
    T = _model_dtype(p)
    a = np.zeros((nblk, 18, 18), np.int32)
    a[:, 1:17, 1:17] = (zb[:, 1:17, 1:17].astype(T) < p.mask).astype(np.int32)
    act = None if a[:, 1:17, 1:17].all() else a
    return dict(zb=zb, zs=zs, h=h, u=np.zeros_like(h), v=np.zeros_like(h), segments=segs, active_cell=act)


def prepare_model(param_file: str, basedir: str | None = None, nblkmem: int | None = None) -> ModelInputs:
    """Steps 1-5 and 7 of the module docstring on the host (no GPU needed).  The
    initial adaptation (step 6) needs the device: ``setup_model`` runs it."""
    basedir = basedir if basedir is not None else os.path.dirname(os.path.abspath(param_file))
    p = read_param_file(param_file)
    if not p.bathy:
        raise ValueError("no bathymetry file specified (bathy = file.asc)")
    if len(p.bathy) > 1:
        raise ValueError("several bathymetry layers are not supported by this library")
    reftime = [p.reftime]
    bathy = read_bathy(_resolve(p.bathy[0], basedir), p.posdown, first=True)
    _boundary_series(p, basedir, reftime)
    rivers = _river_series(p, basedir, reftime)
    rain = _rain_series(p, basedir, reftime)
    outt = check_param_sanity(p, bathy, rain is not None)
    nx, ny, levdx = _mesh_counts(p)
    nbx, nby = -(-nx // 16), -(-ny // 16)
    pres = np.zeros(nbx * nby, np.uint8)
    nkeep = ctypes.c_int(0)
    g = bathy.to_c()
    if lib().bgf_mask_blocks(ctypes.byref(g), nbx, nby, float(p.xo), float(p.yo), float(levdx), float(p.mask),
                             pres.ctypes.data, ctypes.byref(nkeep)) != 0:
        raise ValueError(f"bgf_mask_blocks: {lib().bgf_last_error().decode()}")
    if nkeep.value == 0:
        raise ValueError("every block lies above mask: nothing to compute")
    mesh = uniform_mesh(nbx * 16, nby * 16, levdx, present=pres.reshape(nby, nbx),
                        doubleprecision=bool(p.doubleprecision))
    if p.initlevel != 0:
        mesh.level[:] = p.initlevel
    ic = _initial_conditions(p, bathy, mesh, mesh.level, mesh.nbr, mesh.xo, mesh.yo)
    nmem = nblkmem if nblkmem is not None else int(math.ceil(mesh.nblk * p.membuffer))
    nextout = min(outt[1], p.endtime) if len(outt) > 1 else p.endtime
    return ModelInputs(p, bathy, mesh, ic["zb"], ic["h"], ic["u"], ic["v"], ic["zs"], ic["active_cell"],
                       ic["segments"], rain, rivers, outt, p.totaltime, nextout, max(nmem, mesh.nblk))


def _load(inp: ModelInputs, nblkmem: int):
    from .flow import FlowB200
    f = FlowB200(inp.param, nblkmem)
    m = inp.mesh
    f.set_blocks(m.active, m.level, m.nbr, m.xo, m.yo)
    f.set_bed(_pad(inp.zb, nblkmem), activeCell=None if inp.active_cell is None else _pad(inp.active_cell, nblkmem))
    for typ, times, levels, sides in inp.segments:
        f.add_segment(typ, times, levels, sides)
    if inp.rain is not None:
        f.set_rain(inp.rain[0], inp.rain[1])
    for xs, xe, ys, ye, t, q in inp.rivers:
        f.add_river(xs, xe, ys, ye, t, q)
    f.set_state(_pad(inp.h, nblkmem), _pad(inp.u, nblkmem), _pad(inp.v, nblkmem))
    return f


def _pad(a: np.ndarray, n: int) -> np.ndarray:
    out = np.zeros((n,) + a.shape[1:], a.dtype)
    out[: a.shape[0]] = a
    return out


def inputs_on_mesh(inp: ModelInputs, level, nbr, xo, yo) -> ModelInputs:
    """Step 5 again on other block tables (blocks 0..n-1 in active order, nbr (n, 8),
    origins relative to the domain origin), as InitialAdaptation reruns
    InitialConditions on the refined mesh."""
    n = len(level)
    mesh = Mesh(inp.mesh.nbx, inp.mesh.nby, inp.mesh.dx, n, np.asarray(level, np.int32),
                np.asarray(nbr, np.int32).reshape(n, 8), np.asarray(xo, np.float64), np.asarray(yo, np.float64),
                np.zeros(n, np.int32), np.zeros(n, np.int32))
    ic = _initial_conditions(inp.param, inp.bathy, mesh, mesh.level, mesh.nbr, mesh.xo, mesh.yo)
    return ModelInputs(inp.param, inp.bathy, mesh, ic["zb"], ic["h"], ic["u"], ic["v"], ic["zs"], ic["active_cell"],
                       ic["segments"], inp.rain, inp.rivers, inp.output_times, inp.totaltime, inp.nextoutputtime,
                       max(inp.nblkmem, n), adapted=True)


def _adapted_inputs(inp: ModelInputs, f) -> ModelInputs:
    act, lev, nb, xo, yo = f.get_blocks()
    n = len(act)
    # the tables renumbered to active-list order
    remap = np.full(f.nblkmem, -1, np.int64)
    remap[act] = np.arange(n)
    return inputs_on_mesh(inp, lev[act], remap[nb[act]].astype(np.int32), xo[act], yo[act])


def setup_model(param_file: str, basedir: str | None = None, nblkmem: int | None = None):
    """The scenario of a BG_param.txt on the GPU: returns (FlowB200, ModelInputs, Loop)
    with the loop after InitLoop and initdt, ready for ``FlowB200.run``."""
    from .adapt import parse_criterion
    from .flow import Loop
    inp = prepare_model(param_file, basedir, nblkmem)
    p = inp.param
    if p.maxlevel != p.minlevel:
        if not p.AdaptCrit:
            raise ValueError("maxlevel != minlevel needs an Adaptation criterion")
        cap = nblkmem if nblkmem is not None else max(inp.nblkmem, inp.mesh.nblk * 4 ** (p.maxlevel - p.initlevel))
        f = _load(inp, cap)
        f.set_bathy(inp.bathy.xo, inp.bathy.yo, inp.bathy.dx, inp.bathy.val)
        crit = parse_criterion(",".join([p.AdaptCrit] + list(p.Adapt_args)))
        for fn in crit.maps:
            # a target-level map (readstaticforcing into StaticForcingP<int>): the
            # grid's values truncated to integers, as the int conversion does
            g = read_asc(_resolve(fn, basedir or os.path.dirname(os.path.abspath(param_file))))
            f.add_target_level_map(g.xo, g.yo, g.dx, np.trunc(g.val).astype(np.int32))
        f.adapt(crit, p.adaptmaxiteration)
        inp = _adapted_inputs(inp, f)
        f.close()
        inp.nblkmem = cap
    f = _load(inp, max(inp.nblkmem, inp.mesh.nblk))
    if inp.param.maxlevel != inp.param.minlevel:
        f.set_bathy(inp.bathy.xo, inp.bathy.yo, inp.bathy.dx, inp.bathy.val)
    loop = Loop(totaltime=inp.totaltime, nextoutputtime=inp.output_times[0] if inp.output_times else p.endtime)
    f.init_dt(loop)
    loop.nextoutputtime = inp.nextoutputtime
    return f, inp, loop
