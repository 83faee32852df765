"""The thread layouts of the fused single-level kernels (bgf_set_kernel_layout: one
cell per thread, two cells per thread, or two cells per thread in persistent CTAs
whose producer warp stages each block's tile with bulk asynchronous copies) give
the same results: bit for bit in the exact build, within the fast-math tolerance in
the fast build (there the two-cell kernels use paired FP32 instructions and
contract other products into fused multiply-adds).  All run through the C ABI on
the same inputs, handles and pools."""
import numpy as np
import pytest

import cases
from runners import interior, make_gpu

pytestmark = pytest.mark.gpu

CASES = [
    ("gauss48_e1_b3", lambda: cases.gauss(48, 1, 3), 40),
    ("gauss48_e2_b3", lambda: cases.gauss(48, 2, 3), 40),
    ("hump64_e2", lambda: cases.hump_walls(64, 2), 30),
    ("dam48_e1", lambda: cases.dam_break(48, 1), 40),
    ("dam32_e2", lambda: cases.dam_break(32, 2), 40),
    ("island64_e1", lambda: cases.conical_island(64, 1), 40),
    ("island48_e2", lambda: cases.conical_island(48, 2), 40),
    ("rain48_e1", lambda: cases.rain_on_terrain(48, 1), 30),
]
FAST_TOL = 2e-4      # m, m/s after the stated number of steps
FAST_DT_RTOL = 1e-4


def _run(mk, layout, fast, nsteps, dbl=False):
    case = mk()
    case.param.fastmath = fast
    case.param.doubleprecision = 1 if dbl else 0
    f, _, loop = make_gpu(case)
    f.set_kernel_layout(layout)
    dts = []
    for _ in range(nsteps):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        dts.append(dt)
    return dts, f.get_state()


@pytest.mark.parametrize("layout", [2, 3])
@pytest.mark.parametrize("name,mk,nsteps", CASES, ids=[c[0] for c in CASES])
def test_layouts_bit_identical_exact(name, mk, nsteps, layout):
    d1, s1 = _run(mk, 1, 0, nsteps)
    d2, s2 = _run(mk, layout, 0, nsteps)
    assert d1 == d2
    for k, a, b in zip("zs h u v".split(), s1, s2):
        assert np.array_equal(interior(a), interior(b)), (k, float(np.abs(interior(a) - interior(b)).max()))


@pytest.mark.parametrize("layout", [2, 3])
@pytest.mark.parametrize("name,mk,nsteps", CASES, ids=[c[0] for c in CASES])
def test_layouts_close_fast(name, mk, nsteps, layout):
    d1, s1 = _run(mk, 1, 1, nsteps)
    d2, s2 = _run(mk, layout, 1, nsteps)
    for a, b in zip(d1, d2):
        assert abs(a - b) <= FAST_DT_RTOL * a
    for k, a, b in zip("zs h u v".split(), s1, s2):
        assert float(np.abs(interior(a).astype(np.float64) - interior(b)).max()) <= FAST_TOL, k


@pytest.mark.parametrize("layout", [2, 3])
def test_layouts_bit_identical_double(layout):
    mk = lambda: cases.dam_break(32, 1)
    d1, s1 = _run(mk, 1, 0, 30, dbl=True)
    d2, s2 = _run(mk, layout, 0, 30, dbl=True)
    assert d1 == d2
    for a, b in zip(s1, s2):
        assert np.array_equal(interior(a), interior(b))


@pytest.mark.parametrize("grid", [0, 7])
def test_staged_layout_persistent_grids(grid):
    """The staged kernels with their default resident grid and with 7 CTAs (many
    blocks per CTA, so every CTA refills its stage many times)."""
    mk = lambda: cases.conical_island(128, 1)
    d1, s1 = _run(mk, 1, 0, 25)
    case = mk()
    f, _, loop = make_gpu(case)
    f.set_kernel_layout(3)
    f.set_grid(grid)
    d3 = []
    for _ in range(25):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        d3.append(dt)
    assert d1 == d3
    for a, b in zip(s1, f.get_state()):
        assert np.array_equal(interior(a), interior(b))


def test_staged_layout_in_a_pool():
    """Scenarios of different sizes and step budgets in one pool with the staged
    kernels (finished scenarios stop swapping their state buffers while others run)
    end as each does alone with one cell per thread."""
    from bg_flood_b200.pool import ScenarioPool
    mks = [lambda: cases.gauss(48, 1, 3), lambda: cases.conical_island(64, 1), lambda: cases.dam_break(48, 1)]
    budgets = [17, 30, 23]
    alone = []
    for mk, n in zip(mks, budgets):
        _, st = _run(mk, 1, 0, n)
        alone.append(st)
    built = [make_gpu(mk()) for mk in mks]
    pool = ScenarioPool(mks[0]().param, sum(b[1].nblk for b in built), 4)
    pool.set_kernel_layout(3)
    slots = [pool.admit(f, lp, 1e30, maxsteps=n) for (f, _, lp), n in zip(built, budgets)]
    assert pool.run(64) == 0
    for slot, (f, m, _), st in zip(slots, built, alone):
        h = pool.depth(slot, m.nblk)
        assert np.array_equal(h, interior(st[1])[: m.nblk])
    pool.close()


def test_layout_rejects_other_values():
    f, _, _ = make_gpu(cases.hump_walls(32, 2))
    from bg_flood_b200.flow import BGFError
    for bad in (0, 4):
        with pytest.raises(BGFError):
            f.set_kernel_layout(bad)


# ---------------------------------------------------------------- split precision

def _split(mk):
    def make():
        case = mk()
        case.param.splitprecision = 1
        return case
    return make


SPLIT_CASES = [
    ("tsunami3", _split(lambda: cases.ensemble_member(3, 2024, 64, 512)), 40),
    ("tsunami7", _split(lambda: cases.ensemble_member(7, 2024, 64, 512)), 40),
    ("island64_e1", _split(lambda: cases.conical_island(64, 1)), 40),
    ("hump64_e2", _split(lambda: cases.hump_walls(64, 2)), 30),
    ("rain48_e1", _split(lambda: cases.rain_on_terrain(48, 1)), 30),
]


@pytest.mark.parametrize("name,mk,nsteps", SPLIT_CASES, ids=[c[0] for c in SPLIT_CASES])
def test_split_layouts_bit_identical_exact(name, mk, nsteps):
    """Split precision (FP32 deviations from per-block datums) in the two-cell kernels
    reproduces the one-cell split kernels bit for bit in the exact build: datum
    conversion of neighbour cells, full depths in the wet tests, the limiter and
    friction, and the datum's pressure shift."""
    d1, s1 = _run(mk, 1, 0, nsteps)
    d2, s2 = _run(mk, 2, 0, nsteps)
    assert d1 == d2
    for k, a, b in zip("zs h u v".split(), s1, s2):
        assert np.array_equal(interior(a), interior(b)), (k, float(np.abs(interior(a) - interior(b)).max()))


@pytest.mark.parametrize("name,mk,nsteps", SPLIT_CASES, ids=[c[0] for c in SPLIT_CASES])
def test_split_layouts_close_fast(name, mk, nsteps):
    d1, s1 = _run(mk, 1, 1, nsteps)
    d2, s2 = _run(mk, 2, 1, nsteps)
    for a, b in zip(d1, d2):
        assert abs(a - b) <= FAST_DT_RTOL * a
    for k, a, b in zip("zs h u v".split(), s1, s2):
        assert float(np.abs(interior(a).astype(np.float64) - interior(b)).max()) <= FAST_TOL, k


def test_split_pool_equals_alone():
    """Two split-precision tsunami members batched in one pool (two-cell kernels,
    per-block datums in the pool's slots) end exactly as each does alone."""
    from bg_flood_b200.pool import ScenarioPool
    mks = [SPLIT_CASES[0][1], SPLIT_CASES[1][1]]
    ref = []
    for mk in mks:
        f, mesh, loop = make_gpu(mk())
        n = f.run(loop, endtime=1e30, maxsteps=30)
        ref.append((f.get_state(), loop, n, mesh.nblk))
    pool = ScenarioPool(mks[0]().param, sum(r[3] for r in ref), 2)
    slots = []
    for mk in mks:
        f, mesh, loop = make_gpu(mk())
        slots.append((pool.admit(f, loop, 1e30, maxsteps=30), mesh.nblk))
    assert pool.run(1000) == 0
    for (s, nblk), (st, loop_a, n_a, _) in zip(slots, ref):
        loop, status, n = pool.query(s)
        assert n == n_a == 30 and loop.totaltime == loop_a.totaltime
        # full depths D + h' (the handle forms the sum in FP64, the pool in FP32: both
        # round the same exact sum to FP32)
        got = np.asarray(pool.depth(s, nblk), np.float64).astype(np.float32)
        assert np.array_equal(got, interior(st[1])[:nblk].astype(np.float32))
    pool.close()
