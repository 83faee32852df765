"""GPU parity on multi-level meshes: the sm_100a multi-level step chain through the
C ABI against the CPU oracle on block tables produced by the reference's own
adaptation (tests/golden/amr*.npz).

The exact kernels reproduce the oracle bit for bit (dt sequence and h, u, v);
the fast-math kernels stay within the tolerance written below."""
import os

import numpy as np
import pytest

import cases
from runners import interior, make_gpu_amr, make_oracle_amr

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

FIXTURES = {
    "amrhump64_e1_l1": (lambda: cases.amr_hump(64, 1, 1, 0.3), 30),
    "amrhump64_e2_l2": (lambda: cases.amr_hump(64, 2, 2, 0.3), 30),
    "amrdam64_e1_l2": (lambda: cases.amr_dambreak(64, 1, 2), 40),
    "amrdam64_e2_l2": (lambda: cases.amr_dambreak(64, 2, 2), 40),
    "amrdam64_e1_l3": (lambda: cases.amr_dambreak(64, 1, 3), 40),
}
FAST_FIELD_TOL = 2e-4   # m, m/s after the stated number of steps
FAST_DT_RTOL = 1e-4


def tables(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return g, (g["level"], g["nbr"], g["xo"], g["yo"])


@pytest.mark.parametrize("name", list(FIXTURES))
def test_amr_step_bitexact_vs_oracle(name):
    mk, nsteps = FIXTURES[name]
    g, tab = tables(name)
    f, loop = make_gpu_amr(mk(), tab)
    o = make_oracle_amr(mk(), tab)
    for s in range(nsteps):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert dt == do, (s, dt, do)
    zs, h, u, v = f.get_state()
    for k, a in (("h", h), ("u", u), ("v", v)):
        assert np.array_equal(interior(a), interior(o.get(k)).astype(a.dtype)), (k, float(
            np.abs(interior(a) - interior(o.get(k))).max()))
    # and the reference's own result on the same tables
    for k, a in (("h", h), ("u", u), ("v", v)):
        assert np.array_equal(interior(a).astype(np.float32), g[k]), k


@pytest.mark.parametrize("name", ["amrhump64_e2_l2", "amrdam64_e1_l3"])
def test_amr_device_loop_equals_single_steps(name):
    mk, nsteps = FIXTURES[name]
    _, tab = tables(name)
    f1, l1 = make_gpu_amr(mk(), tab)
    f2, l2 = make_gpu_amr(mk(), tab)
    for _ in range(nsteps):
        l1.totaltime += f1.flow_step(l1)
    n = f2.run(l2, endtime=1e30, maxsteps=nsteps)
    assert n == nsteps
    assert l2.totaltime == l1.totaltime and l2.dt == l1.dt
    for a, b in zip(f1.get_state()[1:], f2.get_state()[1:]):
        assert np.array_equal(interior(a), interior(b))


@pytest.mark.parametrize("name", ["amrhump64_e1_l1", "amrdam64_e2_l2", "amrdam64_e1_l3"])
def test_amr_fastmath_close_to_oracle(name):
    mk, nsteps = FIXTURES[name]
    _, tab = tables(name)
    case = mk()
    case.param.fastmath = 1
    f, loop = make_gpu_amr(case, tab)
    o = make_oracle_amr(mk(), tab)
    for s in range(nsteps):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert abs(dt - do) <= FAST_DT_RTOL * do, (s, dt, do)
    zs, h, u, v = f.get_state()
    for k, a in (("h", h), ("u", u), ("v", v)):
        assert float(np.abs(interior(a).astype(np.float64) - interior(o.get(k))).max()) <= FAST_FIELD_TOL, k


def test_amr_mass_conservation_with_walls():
    """Closed basin on a three-level mesh: the restriction of the coarse/fine fluxes
    keeps the volume constant to float32 round-off over 200 steps."""
    mk, _ = FIXTURES["amrhump64_e2_l2"]
    _, tab = tables("amrhump64_e2_l2")
    f, loop = make_gpu_amr(mk(), tab)
    v0 = f.volume()
    f.run(loop, endtime=1e30, maxsteps=200)
    v1 = f.volume()
    assert abs(v1 - v0) / v0 < 5e-6
