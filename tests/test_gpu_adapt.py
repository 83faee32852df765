"""GPU refinement pass (bgf_adapt) against the reference's own Adaptation() on the
same initial state and bathymetry grid (fixtures tests/golden/adapt_*.npz, written
by tests/golden/make_golden.py).

Bit-exact: the active list, levels, all neighbour tables, block origins, the
re-interpolated bed and the depth h.  u and v: within the tolerance below -- the
reference fills their halos with rules that read a coarser neighbour's halo in
block order, which the device pass evaluates after all halos are filled."""
import os

import numpy as np
import pytest

from adapt_cases import ADAPT_CASES, MEM, criterion_of, level0_grids, target_case, target_maps
from bg_flood_b200.adapt import TARGETLEVEL, Criterion
from bg_flood_b200.flow import FlowB200, Loop
from bg_flood_b200.mesh import boundary_segments, grid_to_buq, uniform_mesh
from runners import interior

pytestmark = pytest.mark.gpu

GOLDEN = os.path.dirname(os.path.abspath(__file__)) + "/golden"
UV_TOL = 1e-5  # m/s


def _pad(a, n):
    out = np.zeros((n, 18, 18), a.dtype)
    out[: len(a)] = a
    return out


def adapted_model(name, steps=0, case=None, maps=()):
    case = case if case is not None else ADAPT_CASES[name]()
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
    if steps:
        loop = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=case.nextoutputtime)
        f.init_dt(loop)
        for _ in range(steps):
            loop.totaltime += f.flow_step(loop)
    for xo, yo, dx, lv in maps:
        f.add_target_level_map(xo, yo, dx, lv)
    crit = Criterion(TARGETLEVEL, "h", 0.0) if maps else criterion_of(case)
    n, it = f.adapt(crit)
    return case, f, n, it


@pytest.mark.parametrize("name,steps", [("island64_e1_l2", 0), ("hump64_e1_l2", 0), ("dam64_e1_l3", 0),
                                        ("hump64_e1_l2", 20), ("island64_e1_l2", 20)])
def test_adaptation_matches_reference(name, steps):
    """steps > 0: adaptation in the middle of a run (the flow steps before it are
    bit-exact with the reference, so both adapt the same state)."""
    g = np.load(os.path.join(GOLDEN, f"adapt_{name}{'_t%d' % steps if steps else ''}.npz"))
    case, f, n, it = adapted_model(name, steps)
    act, lev, nb, xo, yo = f.get_blocks()
    assert n == len(g["act"]) and it >= 1
    assert np.array_equal(act, g["act"])
    assert np.array_equal(lev[act], g["level"])
    assert np.array_equal(nb[act], g["nbr"])
    assert np.array_equal(xo[act].astype(np.float32), g["xo"].astype(np.float32))
    assert np.array_equal(yo[act].astype(np.float32), g["yo"].astype(np.float32))
    zb = interior(f.get_bed()[act])
    assert np.array_equal(zb, g["zb"])
    zs, h, u, v = f.get_state()
    assert np.array_equal(interior(h[act]), g["h"])
    assert float(np.abs(interior(u[act]) - g["u"]).max()) <= UV_TOL
    assert float(np.abs(interior(v[act]) - g["v"]).max()) <= UV_TOL


def test_targetlevel_adaptation_matches_reference():
    """Targetlevel with two maps, the second overriding the first (the reference's
    Adaptation() with the same maps: tests/golden/adapt_target_hump64.npz)."""
    g = np.load(os.path.join(GOLDEN, "adapt_target_hump64.npz"))
    case = target_case()
    case, f, n, it = adapted_model("target", case=case, maps=target_maps(case))
    act, lev, nb, xo, yo = f.get_blocks()
    assert n == len(g["act"]) and set(np.unique(lev[act])) == {0, 1, 2}
    assert np.array_equal(act, g["act"])
    assert np.array_equal(lev[act], g["level"])
    assert np.array_equal(nb[act], g["nbr"])
    assert np.array_equal(xo[act].astype(np.float32), g["xo"].astype(np.float32))
    assert np.array_equal(yo[act].astype(np.float32), g["yo"].astype(np.float32))
    assert np.array_equal(interior(f.get_bed()[act]), g["zb"])
    zs, h, u, v = f.get_state()
    assert np.array_equal(interior(h[act]), g["h"])
    # without a map the criterion is refused
    f.clear_target_level_maps()
    with pytest.raises(Exception):
        f.adapt(Criterion(TARGETLEVEL, "h", 0.0))


def test_adapted_mesh_steps_on_multilevel_path():
    """The adapted handle runs the multi-level step and conserves volume with walls."""
    case, f, n, it = adapted_model("hump64_e1_l2")
    loop = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=case.nextoutputtime)
    f.init_dt(loop)
    v0 = f.volume()
    f.run(loop, endtime=1e30, maxsteps=100)
    assert abs(f.volume() - v0) / v0 < 5e-6
