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
    mesh = mesh or uniform_mesh(case.nx, case.ny, case.dx)
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


def make_reference(case: Case, use_double: bool = False) -> Reference:
    r = Reference(case.paramtext, case.nx, case.ny, case.dx, case.xo, case.yo, case.zb, case.h, case.u, case.v,
                  case.cf, case.nextoutputtime, use_double)
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
