"""Drivers that run one Case through the reference, the oracle and the GPU library
with identical inputs (test infrastructure)."""
from __future__ import annotations

import numpy as np

from bg_flood_b200.mesh import boundary_segments, fill_halo, grid_to_buq, uniform_mesh
from cases import Case
from oracle.pyoracle import Oracle, Reference

INTERIOR = (slice(None), slice(1, 17), slice(1, 17))


def interior(a: np.ndarray) -> np.ndarray:
    return np.asarray(a).reshape(-1, 18, 18)[INTERIOR]


def make_oracle(case: Case, use_double: bool = False, mesh=None):
    mesh = mesh or uniform_mesh(case.nx, case.ny, case.dx, doubleprecision=use_double)
    o = Oracle(case.param, mesh.nblk, use_double)
    o.set_blocks(mesh.level, mesh.nbr, mesh.xo, mesh.yo)
    o.set("zb", grid_to_buq(case.zb, mesh))
    for name in ("h", "u", "v"):
        o.set(name, grid_to_buq(getattr(case, name), mesh))
    o.set("zs", grid_to_buq((case.zb + case.h).astype(np.float32), mesh))
    if case.cf is not None:
        o.set("cf", grid_to_buq(case.cf, mesh))
    for typ, times, levels, sides in boundary_segments(mesh, case.param.segments, case.param.aoibnd, case.xo, case.yo):
        o.add_segment(typ, times, levels, sides)
    if case.rain is not None:
        o.set_rain(*case.rain)
        from bg_flood_b200.flow import _rain_mask
        act = _rain_mask(grid_to_buq(case.zb, mesh), case.param.mask)
        if act is not None:
            o.set("activeCell", act.astype(np.float64))
    o.init_bed()
    o.init_loop(0.0, case.nextoutputtime)
    return o, mesh


def make_reference(case: Case, use_double: bool = False, lib_path: str | None = None) -> Reference:
    r = Reference(case.paramtext, case.nx, case.ny, case.dx, case.xo, case.yo, case.zb, case.h, case.u, case.v,
                  case.cf, case.nextoutputtime, use_double, lib_path=lib_path)
    for k, seg in enumerate(case.param.segments):
        if seg.times:
            r.set_segment_series(k, seg.times, seg.levels)
    if case.rain is not None:
        r.set_rain(*case.rain)
    return r


def make_gpu(case: Case):
    from bg_flood_b200.flow import Loop, build_model
    f, mesh = build_model(case.param, case.zb, case.h, case.u, case.v, cf=case.cf, rain=case.rain)
    loop = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=case.nextoutputtime)
    f.init_dt(loop)
    return f, mesh, loop


def gpu_fields(f) -> dict:
    zs, h, u, v = f.get_state()
    return {"zs": zs, "h": h, "u": u, "v": v}


def oracle_fields(o: Oracle) -> dict:
    return {k: o.get(k) for k in ("zs", "h", "u", "v")}


def maxdiff(a, b) -> float:
    return float(np.max(np.abs(interior(a).astype(np.float64) - interior(b).astype(np.float64))))


def _sample(fn, level, xo, yo, case, zb=None):
    """fn at the cell centres of every block (tiles (nblk, 18, 18), halo left 0)."""
    n = len(level)
    out = np.zeros((n, 18, 18))
    ii = np.arange(16)
    for b in range(n):
        d = case.dx / (2.0 ** level[b])
        X, Y = np.meshgrid(case.xo + xo[b] + ii * d, case.yo + yo[b] + ii * d)
        out[b, 1:17, 1:17] = fn(X, Y) if zb is None else fn(X, Y, zb[b, 1:17, 1:17])
    return out.astype(np.float32).astype(np.float64)


def amr_fields(case, lev, xo, yo):
    """Bed and depth of an AMR case sampled at the cell centres of the given blocks."""
    zb = _sample(case.zb_fn, lev, xo, yo, case)
    h = _sample(lambda X, Y, Z: np.maximum(case.eta_fn(X, Y) - Z, 0.0), lev, xo, yo, case, zb=zb)
    return zb, h


def amr_mesh(case, lev, nbr, xo, yo):
    from bg_flood_b200.mesh import Mesh
    n = len(lev)
    return Mesh(case.n0 // 16, case.n0 // 16, case.dx, n, np.asarray(lev, np.int32), np.asarray(nbr, np.int32),
                np.asarray(xo), np.asarray(yo), np.zeros(n, np.int32), np.zeros(n, np.int32))


def make_oracle_amr(case, tables, use_double: bool = False):
    """The oracle on given block tables (level, nbr (n, 8), xo, yo) of an AMR case."""
    lev, nbr, xo, yo = tables
    zb, h = amr_fields(case, lev, xo, yo)
    zero = np.zeros_like(zb)
    o = Oracle(case.param, len(lev), use_double)
    o.set_blocks(lev, nbr, xo, yo)
    for name, a in (("zb", zb), ("h", h), ("u", zero), ("v", zero)):
        o.set(name, a)
    o.set("zs", (zb + h).astype(np.float32))
    m = amr_mesh(case, lev, nbr, xo, yo)
    for typ, times, levels, sides in boundary_segments(m, case.param.segments, case.param.aoibnd, case.xo, case.yo):
        o.add_segment(typ, times, levels, sides)
    o.init_bed()
    o.init_loop(0.0, case.nextoutputtime)
    return o


def make_gpu_amr(case, tables):
    """The GPU library on given block tables of an AMR case; returns (FlowB200, Loop)."""
    from bg_flood_b200.flow import FlowB200, Loop
    lev, nbr, xo, yo = tables
    zb, h = amr_fields(case, lev, xo, yo)
    zero = np.zeros_like(zb)
    n = len(lev)
    f = FlowB200(case.param, n)
    f.set_blocks(np.arange(n, dtype=np.int32), lev, nbr, xo, yo)
    f.set_bed(zb)
    m = amr_mesh(case, lev, nbr, xo, yo)
    for typ, times, levels, sides in boundary_segments(m, case.param.segments, case.param.aoibnd, case.xo, case.yo):
        f.add_segment(typ, times, levels, sides)
    f.set_state(h, zero, zero)
    loop = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=case.nextoutputtime)
    f.init_dt(loop)
    return f, loop


def make_amr_pair(case):
    """The reference adapts the mesh; the oracle gets the same tables and fields.
    Returns (reference, oracle, (level, nbr, xo, yo))."""
    n0 = case.n0
    ii = (np.arange(n0) + 0.5) * case.dx
    X, Y = np.meshgrid(case.xo + ii, case.yo + ii)
    zb0 = case.zb_fn(X, Y).astype(np.float32)
    eta0 = case.adapt_eta_fn if case.adapt_eta_fn is not None else case.eta_fn
    h0 = np.maximum(eta0(X, Y) - zb0, 0).astype(np.float32)
    z0 = np.zeros_like(zb0)
    r = Reference(case.paramtext, n0, n0, case.dx, case.xo, case.yo, zb0, h0, z0, z0, None, case.nextoutputtime)
    r.adapt()
    tables = r.mesh_active_order()
    lev, nbr, xo, yo = tables
    zb, h = amr_fields(case, lev, xo, yo)
    zero = np.zeros_like(zb)
    for name, a in (("zb", zb), ("h", h), ("u", zero), ("v", zero)):
        r.set(name, a)
    r.reinit(case.nextoutputtime)
    return r, make_oracle_amr(case, tables), tables


def make_oracle_inputs(inp):
    """The oracle on a scenario set up from its input files (bg_flood_b200.model_setup
    ModelInputs): same tables, bed, state (zs = zb + h), segments, rain and mask,
    the loop as InitLoop and the first map output leave it."""
    p = inp.param
    m = inp.mesh
    dbl = bool(p.doubleprecision)
    o = Oracle(p, m.nblk, dbl)
    o.set_blocks(m.level, m.nbr, m.xo, m.yo)
    T = np.float64 if dbl else np.float32
    zb = inp.zb.astype(T)
    h = inp.h.astype(T)
    for name, a in (("zb", zb), ("h", h), ("u", inp.u), ("v", inp.v)):
        o.set(name, a)
    o.set("zs", (zb + h).astype(T))
    if inp.active_cell is not None:
        o.set("activeCell", inp.active_cell)
    for typ, times, levels, sides in inp.segments:
        o.add_segment(typ, times, levels, sides)
    if inp.rain is not None:
        o.set_rain(inp.rain[0], inp.rain[1])
    for xs, xe, ys, ye, t, q in inp.rivers:
        o.add_river(xs, xe, ys, ye, t, q)
    o.init_bed()
    dtmax = o.init_loop(inp.totaltime, inp.output_times[0])
    o.set_loop(inp.totaltime, inp.nextoutputtime, dtmax)
    return o


def normalise_reference_surface(ref, dbl: bool) -> None:
    """Sets the reference's initial zs to zb + h (in the model precision), the
    surface this library's state implies, before stepping it."""
    T = np.float64 if dbl else np.float32
    zb, h, zs = ref.get("zb"), ref.get("h"), ref.get("zs")
    zs[:, 1:17, 1:17] = (zb[:, 1:17, 1:17].astype(T) + h[:, 1:17, 1:17].astype(T)).astype(np.float64)
    ref.set("zs", zs)
