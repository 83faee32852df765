"""GPU refinement pass with the coarsening extension (bgf_adapt, allow_coarsen) and
the depth-or-slope criterion, against the CPU restatement in coarsen_restate.py:

* criterion flags and sanity-pass flags, bit for bit;
* block tables after a pass equal bgf_adapt_tables applied to those flags (the
  table function is checked against mesh invariants on the CPU);
* the merged parents' h, u, v equal the quad means of the old cells followed by the
  reference's wet/dry fix-up on the re-interpolated bed (src/Adaptation.cu:690-770,
  500-525), bit for bit;
* the coarsened mesh then steps bit for bit with the oracle on the same tables."""
import numpy as np
import pytest

import cases
import coarsen_restate as cr
from adapt_cases import level0_grids
from bg_flood_b200.adapt import adapt_tables, depth_or_slope
from bg_flood_b200.flow import FlowB200, Loop
from bg_flood_b200.mesh import boundary_segments, grid_to_buq, uniform_mesh
from oracle.pyoracle import Oracle
from runners import amr_mesh, interior

pytestmark = pytest.mark.gpu

MEM = 2048


def _pad(a, n):
    out = np.zeros((n, 18, 18), a.dtype)
    out[: len(a)] = a
    return out


def dam_handle():
    """Level-0 64x64 dam break (engine 1, maxlevel 3) with its bathymetry grid."""
    case = cases.amr_dambreak(64, 1, 3)
    zb0, h0 = level0_grids(case)
    mesh = uniform_mesh(case.n0, case.n0, case.dx)
    f = FlowB200(case.param, MEM)
    f.set_blocks(mesh.active, mesh.level, mesh.nbr, mesh.xo, mesh.yo)
    f.set_bed(_pad(grid_to_buq(zb0, mesh), MEM))
    for typ, times, levels, sides in boundary_segments(mesh, case.param.segments, case.param.aoibnd, case.xo, case.yo):
        f.add_segment(typ, times, levels, sides)
    z = np.zeros_like(h0)
    f.set_state(*(_pad(grid_to_buq(a, mesh), MEM) for a in (h0, z, z)))
    f.set_bathy(case.xo + 0.5 * case.dx, case.yo + 0.5 * case.dx, case.dx, zb0)
    return case, f


def snapshot(f):
    act, lev, nbr, xo, yo = f.get_blocks()
    zs, h, u, v = f.get_state()
    zb = f.get_bed()
    hi = interior(h).astype(np.float32)
    zsi = (interior(zb).astype(np.float32) + hi).astype(np.float32)  # zs as the pass takes it: zb + h
    return dict(act=act.copy(), lev=lev.copy(), nbr=nbr.copy(), xo=xo.copy(), yo=yo.copy(), h=hi, zs=zsi,
                u=interior(u).astype(np.float32), v=interior(v).astype(np.float32), zb=zb)


def expected_flags(case, s, crit, allow):
    r, c = cr.hgrad_flags(s["h"], s["zs"], s["lev"], s["act"], case.dx, case.param.eps, crit.arg1, crit.arg2)
    return cr.sanity(s["act"], s["lev"], s["nbr"], case.param.minlevel, case.param.maxlevel, s["xo"], s["yo"],
                     case.dx, r, c, allow_coarsen=allow)


def run_steps(f, case, n):
    loop = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=case.nextoutputtime)
    f.init_dt(loop)
    for _ in range(n):
        loop.totaltime += f.flow_step(loop)


def refined_then_run(steps=40):
    case, f = dam_handle()
    n, it = f.adapt(depth_or_slope(0.3, 0.05), maxiteration=3)
    assert n > 16
    run_steps(f, case, steps)
    return case, f


@pytest.mark.parametrize("allow", [False, True])
def test_depth_or_slope_flags_match_restatement(allow):
    case, f = refined_then_run(30)
    s = snapshot(f)
    for crit in (depth_or_slope(0.3, 0.05), depth_or_slope(2.0, 0.5), depth_or_slope(0.6, 0.02)):
        r, c = f.adapt_flags(crit, allow_coarsen=allow)
        er, ec = expected_flags(case, s, crit, allow)
        assert np.array_equal(r, er[s["act"]]), crit
        assert np.array_equal(c, ec[s["act"]]), crit


def test_coarsening_pass_matches_restatement():
    case, f = refined_then_run(40)
    s = snapshot(f)
    # every block is a candidate (h <= 5 m, slope <= 50): the level-3 quads of the wet
    # region merge wherever no finer block borders them
    crit = depth_or_slope(10.0, 100.0)
    er, ec = expected_flags(case, s, crit, True)
    assert ec[s["act"]].any(), "the case must merge some quads"
    mem = f.nblkmem
    t = adapt_tables(s["act"], s["lev"], s["nbr"].reshape(mem, 8), s["xo"], s["yo"], mem, case.dx, 0, er, ec)
    act2, lev2, nbr2, x2, y2, ch, sb = t
    n, it = f.adapt(crit, maxiteration=1, allow_coarsen=True)
    a, lv, nb, xo, yo = f.get_blocks()
    assert n == len(act2) and np.array_equal(a, act2)
    assert np.array_equal(lv[a], lev2[a]) and np.array_equal(nb[a], nbr2[a])
    assert np.array_equal(xo[a], x2[a]) and np.array_equal(yo[a], y2[a])
    # merged parents: quad means, then the wet/dry fix-up on the new bed
    quads = [(p, *sb[p]) for p in s["act"] if sb[p, 0] >= 0]
    assert quads
    zs, h, u, v = f.get_state()
    zb = interior(f.get_bed()).astype(np.float32)
    eps = np.float32(case.param.eps)
    mh, mzs, mu, mv = (cr.merged_cells(s[k], quads) for k in ("h", "zs", "u", "v"))
    for q in quads:
        p = q[0]
        hm = mh[p]
        wet = hm.astype(np.float64) > case.param.eps
        hexp = np.where(wet, np.maximum(eps, (mzs[p] - zb[p]).astype(np.float32)), hm).astype(np.float32)
        assert np.array_equal(interior(h)[p].astype(np.float32), hexp), p
        assert np.array_equal(interior(u)[p].astype(np.float32), mu[p]), p
        assert np.array_equal(interior(v)[p].astype(np.float32), mv[p]), p
    # blocks the pass left alone keep their state up to the same fix-up (same bed)
    untouched = [ib for ib in a if ib in set(s["act"].tolist()) and sb[ib, 0] < 0 and ch[ib, 0] < 0]
    for ib in untouched:
        hb = s["h"][ib]
        wet = hb.astype(np.float64) > case.param.eps
        hexp = np.where(wet, np.maximum(eps, (s["zs"][ib] - zb[ib]).astype(np.float32)), hb)
        assert np.array_equal(interior(h)[ib].astype(np.float32), hexp.astype(np.float32)), ib
        assert np.array_equal(interior(u)[ib].astype(np.float32), s["u"][ib])


def test_coarsened_mesh_steps_match_oracle():
    case, f = refined_then_run(40)
    f.adapt(depth_or_slope(10.0, 100.0), maxiteration=1, allow_coarsen=True)
    a, lv, nb, xo, yo = f.get_blocks()
    assert (lv[a] < lv[a].max()).any() and len(set(lv[a].tolist())) > 1
    pos = np.full(f.nblkmem, -1, np.int64)
    pos[a] = np.arange(len(a))
    lev_a, nbr_a, xo_a, yo_a = lv[a], pos[nb[a]].astype(np.int32), xo[a], yo[a]
    zs, h, u, v = f.get_state()
    zb = f.get_bed()
    o = Oracle(case.param, len(a))
    o.set_blocks(lev_a, nbr_a, xo_a, yo_a)
    tiles = lambda arr: np.where(np.pad(np.ones((16, 16), bool), 1)[None], arr[a], 0.0).astype(np.float64)
    zbt, ht = tiles(zb), tiles(h)
    for name, arr in (("zb", zbt), ("h", ht), ("u", tiles(u)), ("v", tiles(v))):
        o.set(name, arr)
    o.set("zs", (zbt.astype(np.float32) + ht.astype(np.float32)).astype(np.float64))
    m = amr_mesh(case, lev_a, nbr_a, xo_a, yo_a)
    for typ, times, levels, sides in boundary_segments(m, case.param.segments, case.param.aoibnd, case.xo, case.yo):
        o.add_segment(typ, times, levels, sides)
    o.init_bed()
    o.init_loop(0.0, case.nextoutputtime)
    assert np.array_equal(interior(o.get("zb")).astype(np.float32), interior(zb[a]).astype(np.float32))
    loop = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=case.nextoutputtime)
    f.init_dt(loop)
    for k in range(30):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert dt == do, (k, dt, do)
    zs, h, u, v = f.get_state()
    for name, arr in (("h", h), ("u", u), ("v", v)):
        assert np.array_equal(interior(arr[a]).astype(np.float32), interior(o.get(name)).astype(np.float32)), name
