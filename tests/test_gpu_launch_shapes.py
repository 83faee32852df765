"""Launch shapes of the fused step kernels and the autotuner that picks one.

A persistent grid (fewer CTAs than blocks, each CTA looping over blocks) computes
every block exactly as one CTA per block does, so the results are bit for bit
the same; the autotuner times the shapes from the current state, keeps the
fastest and leaves the state, time slot and maximum depths as they were.
"""
import numpy as np
import pytest

import cases
from bg_flood_b200.pool import ScenarioPool
from runners import interior, make_gpu

pytestmark = pytest.mark.gpu

STEPS = 30
# 20 x 20 blocks: more than 2 CTAs per SM on 148 SMs, so persistent grids are tried
N = 320


def _run(case, grid, steps=STEPS):
    f, mesh, loop = make_gpu(case)
    if grid is not None:
        f.set_grid(grid)
    f.run(loop, endtime=1e30, maxsteps=steps)
    return f, loop


@pytest.mark.parametrize("mk", [lambda: cases.rain_on_terrain(N, 1), lambda: cases.dam_break(N, 2)],
                         ids=["rain_e1", "dam_e2"])
@pytest.mark.parametrize("grid", [148, 296, 444, 1000])
def test_persistent_grid_matches_one_cta_per_block(mk, grid):
    f0, l0 = _run(mk(), 0)
    f1, l1 = _run(mk(), grid)
    assert (l1.totaltime, l1.dt) == (l0.totaltime, l0.dt)
    for a, b in zip(f0.get_state(), f1.get_state()):
        assert np.array_equal(interior(a), interior(b))


def test_autotune_keeps_state_and_picks_a_shape():
    case = cases.rain_on_terrain(N, 1)
    f, mesh, loop = make_gpu(case)
    f.run(loop, endtime=1e30, maxsteps=10)
    before = [interior(a).copy() for a in f.get_state()]
    t0, dt0 = loop.totaltime, loop.dt
    grid, ms = f.autotune(loop, steps=10)
    assert grid == 0 or (grid % 148 == 0 and grid < mesh.nblk)
    assert ms > 0
    assert (loop.totaltime, loop.dt) == (t0, dt0)
    for a, b in zip(before, f.get_state()):
        assert np.array_equal(a, interior(b))
    # the tuned handle continues exactly like an untuned one
    f.run(loop, endtime=1e30, maxsteps=STEPS)
    g, lg = _run(cases.rain_on_terrain(N, 1), None, 10)
    g.run(lg, endtime=1e30, maxsteps=STEPS)
    assert (lg.totaltime, lg.dt) == (loop.totaltime, loop.dt)
    for a, b in zip(g.get_state(), f.get_state()):
        assert np.array_equal(interior(a), interior(b))


def test_pool_autotune_keeps_state():
    mks = [lambda: cases.rain_on_terrain(N, 1), lambda: cases.gauss(256, 1, 3)]
    budgets = [60, 60]
    ref = []
    for mk, n in zip(mks, budgets):
        f, _, loop = make_gpu(mk())
        f.run(loop, endtime=1e30, maxsteps=n)
        ref.append((f.get_state(), loop))
    pool = ScenarioPool(mks[0]().param, 1024, 2, track_hmax=True)
    slots, nblks = [], []
    for mk, n in zip(mks, budgets):
        f, mesh, loop = make_gpu(mk())
        nblks.append(mesh.nblk)
        slots.append(pool.admit(f, loop, 1e30, maxsteps=n))
    pool.run(20)
    depth = [pool.depth(s, nb, with_max=True) for s, nb in zip(slots, nblks)]
    grid, ms = pool.autotune(steps=6)
    assert grid == 0 or grid % 148 == 0
    assert ms > 0
    for s, nb, (h, hm) in zip(slots, nblks, depth):
        h2, hm2 = pool.depth(s, nb, with_max=True)
        assert np.array_equal(h, h2) and np.array_equal(hm, hm2)
    assert pool.run(1000) == 0
    for s, (st, loop_a) in zip(slots, ref):
        f, loop, n = pool.retire(s)
        assert loop.totaltime == loop_a.totaltime and loop.dt == loop_a.dt
        for a, b in zip(f.get_state()[1:], st[1:]):
            assert np.array_equal(interior(a), interior(b))
