"""The two thread layouts of the fused single-level kernels (bgf_set_kernel_layout:
two cells per thread, or one cell per thread) give the same results: bit for bit
in the exact build, within the fast-math tolerance in the fast build (there the
two-cell kernels use paired FP32 instructions and contract other products into
fused multiply-adds).  Both run through the C ABI on the same inputs."""
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


@pytest.mark.parametrize("name,mk,nsteps", CASES, ids=[c[0] for c in CASES])
def test_layouts_bit_identical_exact(name, mk, nsteps):
    d1, s1 = _run(mk, 1, 0, nsteps)
    d2, s2 = _run(mk, 2, 0, nsteps)
    assert d1 == d2
    for k, a, b in zip("zs h u v".split(), s1, s2):
        assert np.array_equal(interior(a), interior(b)), (k, float(np.abs(interior(a) - interior(b)).max()))


@pytest.mark.parametrize("name,mk,nsteps", CASES, ids=[c[0] for c in CASES])
def test_layouts_close_fast(name, mk, nsteps):
    d1, s1 = _run(mk, 1, 1, nsteps)
    d2, s2 = _run(mk, 2, 1, nsteps)
    for a, b in zip(d1, d2):
        assert abs(a - b) <= FAST_DT_RTOL * a
    for k, a, b in zip("zs h u v".split(), s1, s2):
        assert float(np.abs(interior(a).astype(np.float64) - interior(b)).max()) <= FAST_TOL, k


def test_layouts_bit_identical_double():
    mk = lambda: cases.dam_break(32, 1)
    d1, s1 = _run(mk, 1, 0, 30, dbl=True)
    d2, s2 = _run(mk, 2, 0, 30, dbl=True)
    assert d1 == d2
    for a, b in zip(s1, s2):
        assert np.array_equal(interior(a), interior(b))


def test_layout_rejects_other_values():
    f, _, _ = make_gpu(cases.hump_walls(32, 2))
    from bg_flood_b200.flow import BGFError
    with pytest.raises(BGFError):
        f.set_kernel_layout(3)
