"""GPU parity: the sm_100a kernels through the C ABI against the CPU oracle on the
same inputs.

Bit-exact (dt sequence and h, u, v) wherever the reference path uses only IEEE
+ - * / sqrt (the library is built with --fmad=false).  Cases with Manning
friction call cbrtf, which glibc (reference, oracle) and CUDA round differently
in the last place; those are compared with the tolerance written in the test.
"""
import json
import os

import numpy as np
import pytest

import cases
from runners import interior, make_gpu, make_oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

EXACT = [
    ("gauss48_e1_b3", lambda: cases.gauss(48, 1, 3), 40),
    ("gauss48_e2_b3", lambda: cases.gauss(48, 2, 3), 40),
    ("gauss32_e1_b0", lambda: cases.gauss(32, 1, 0), 40),
    ("hump64_e2", lambda: cases.hump_walls(64, 2), 30),
    ("hump48_e1", lambda: cases.hump_walls(48, 1), 30),
    ("dam48_e1", lambda: cases.dam_break(48, 1), 40),
    ("dam32_e2", lambda: cases.dam_break(32, 2), 40),
    ("island64_e1_still", lambda: cases.conical_island(64, 1, wave=False), 20),
]
# Manning friction (cbrtf): relative dt and absolute field tolerances
TOLERANT = [
    ("island64_e1", lambda: cases.conical_island(64, 1), 40),
    ("island48_e2", lambda: cases.conical_island(48, 2), 40),
    ("rain48_e1", lambda: cases.rain_on_terrain(48, 1), 30),
]
FIELD_TOL = 1e-5   # m or m/s after the stated number of steps
DT_RTOL = 1e-5


def _compare(f, o, exact):
    zs, h, u, v = f.get_state()
    for name, a in (("h", h), ("u", u), ("v", v)):
        b = o.get(name)
        ga, gb = interior(a).astype(np.float64), interior(b)
        if exact:
            assert np.array_equal(ga, gb), (name, float(np.abs(ga - gb).max()))
        else:
            assert float(np.abs(ga - gb).max()) <= FIELD_TOL, name


@pytest.mark.parametrize("name,mk,nsteps", EXACT, ids=[c[0] for c in EXACT])
def test_flow_step_bitexact_vs_oracle(name, mk, nsteps):
    case = mk()
    f, mesh, loop = make_gpu(case)
    o, _ = make_oracle(case)
    for s in range(nsteps):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert dt == do, (s, dt, do)
    _compare(f, o, True)
    assert f.kernel_launches() >= 2 * nsteps


@pytest.mark.parametrize("name,mk,nsteps", TOLERANT, ids=[c[0] for c in TOLERANT])
def test_flow_step_close_to_oracle(name, mk, nsteps):
    case = mk()
    f, mesh, loop = make_gpu(case)
    o, _ = make_oracle(case)
    for s in range(nsteps):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert abs(dt - do) <= DT_RTOL * do, (s, dt, do)
    _compare(f, o, False)


@pytest.mark.parametrize("name,mk,nsteps", EXACT, ids=[c[0] for c in EXACT])
def test_device_loop_equals_single_steps(name, mk, nsteps):
    """bgf_run (device-resident loop in CUDA graphs) == nsteps calls of bgf_flow_step
    == the oracle, so that a difference names the path that departs."""
    case = mk()
    f1, _, l1 = make_gpu(case)
    f2, _, l2 = make_gpu(case)
    for _ in range(nsteps):
        l1.totaltime += f1.flow_step(l1)
    n = f2.run(l2, endtime=1e30, maxsteps=nsteps)
    assert n == nsteps
    o, _ = make_oracle(mk())
    o.step(nsteps)
    assert l2.totaltime == l1.totaltime and l2.dt == l1.dt
    for k, a, b in zip("h u v".split(), f1.get_state()[1:], f2.get_state()[1:]):
        ref = interior(o.get(k)).astype(a.dtype)
        assert np.array_equal(interior(a), ref), ("single steps vs oracle", k)
        assert np.array_equal(interior(b), ref), ("device loop vs oracle", k)


def test_device_loop_stops_at_endtime_and_hits_output_times():
    """The device loop clamps dt onto the output times and stops at endtime exactly
    like the oracle driven with the same output schedule."""
    case = cases.hump_walls(64, 2)
    f, _, loop = make_gpu(case)
    o, _ = make_oracle(case)
    o.set_loop(0.0, 2.0, loop.dtmax)
    loop.nextoutputtime = 2.0
    n = f.run(loop, endtime=5.0, outputtimestep=2.0)
    t, steps, next_out = 0.0, 0, 2.0
    while t < 5.0:
        dt = float(o.step(1)[0])
        t = o.totaltime
        steps += 1
        if next_out - t <= dt * 1e-5:
            next_out = min(next_out + 2.0, 5.0)
            o.set_loop(t, next_out, dt)
    assert steps == n
    assert loop.totaltime == t
    zs, h, u, v = f.get_state()
    assert np.array_equal(interior(h), interior(o.get("h")))


@pytest.mark.parametrize("name", ["gauss48_e1_b3", "gauss48_e2_b3", "hump64_e2", "dam48_e1"])
def test_gpu_matches_reference_fixture(name):
    mk = {"gauss48_e1_b3": lambda: cases.gauss(48, 1, 3), "gauss48_e2_b3": lambda: cases.gauss(48, 2, 3),
          "hump64_e2": lambda: cases.hump_walls(64, 2), "dam48_e1": lambda: cases.dam_break(48, 1)}[name]
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    f, _, loop = make_gpu(mk())
    for s in range(int(g["nsteps"])):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        assert dt == g["dts"][s]
    zs, h, u, v = f.get_state()
    for k, a in (("h", h), ("u", u), ("v", v)):
        assert np.array_equal(interior(a).astype(np.float32), g[k]), k


def test_gaussian_hump_known_answer_on_gpu():
    ref = json.load(open(os.path.join(GOLDEN, "zs_verif_buttinger.json")))
    case = cases.gauss(256, engine=1, aoibnd=3)
    f, mesh, loop = make_gpu(case)
    f.run(loop, endtime=0.1)
    zs = f.get_state()[0]
    for k, expect in enumerate(ref["zs"]):
        ii, jj = 16 * (k + 1) - 1, 127
        ib = int(np.flatnonzero((mesh.bx == ii // 16) & (mesh.by == jj // 16))[0])
        assert abs(float(zs[ib, jj % 16 + 1, ii % 16 + 1]) - expect) <= ref["tolerance"]


def test_double_precision_bitexact_vs_oracle():
    case = cases.dam_break(32, 1)
    case.param.doubleprecision = 1
    f, _, loop = make_gpu(case)
    o, _ = make_oracle(case, use_double=True)
    for s in range(30):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        assert dt == o.step(1)[0]
    zs, h, u, v = f.get_state()
    for name, a in (("h", h), ("u", u), ("v", v)):
        assert np.array_equal(interior(a), interior(o.get(name))), name


# ---------------------------------------------------------------- full-size properties

def test_mass_conservation_with_walls_full_size():
    """256x256 hump in a closed basin: volume constant to float32 round-off."""
    case = cases.hump_walls(256, 2)
    f, _, loop = make_gpu(case)
    v0 = f.volume()
    f.run(loop, endtime=10.0)
    v1 = f.volume()
    assert abs(v1 - v0) / v0 < 2e-6


def test_lake_at_rest_is_preserved():
    """Still water around the conical island stays still (well-balanced scheme)."""
    for engine in (1, 2):
        case = cases.conical_island(128, engine, wave=False)
        case.param.frictionmodel = 0
        case.param.cf = 0.0
        f, _, loop = make_gpu(case)
        f.run(loop, endtime=2.0)
        zs, h, u, v = f.get_state()
        assert float(np.abs(interior(u)).max()) < 1e-5
        assert float(np.abs(interior(v)).max()) < 1e-5


def test_symmetric_hump_stays_symmetric():
    """Engine 2 on a centred hump: the X and Y sweeps are the same formula, so the
    solution is symmetric under x <-> y up to the summation order of the flux
    divergence (X then Y terms), i.e. to float32 rounding."""
    from bg_flood_b200.mesh import buq_to_grid
    case = cases.hump_walls(128, 2)
    f, mesh, loop = make_gpu(case)
    f.run(loop, endtime=5.0)
    zs, h, u, v = f.get_state()
    H = buq_to_grid(h, mesh)
    U = buq_to_grid(u, mesh)
    V = buq_to_grid(v, mesh)
    assert float(np.abs(H - H.T).max()) <= 1e-6 * float(np.abs(H).max())
    assert float(np.abs(U - V.T).max()) <= 1e-5 * float(np.abs(U).max())


# ---------------------------------------------------------------- fast-math kernels

FAST_CASES = [
    ("gauss48_e1_b3", lambda: cases.gauss(48, 1, 3), 40),
    ("hump64_e2", lambda: cases.hump_walls(64, 2), 30),
    ("dam48_e1", lambda: cases.dam_break(48, 1), 40),
    ("island64_e1", lambda: cases.conical_island(64, 1), 40),
    ("rain48_e1", lambda: cases.rain_on_terrain(48, 1), 30),
]
FAST_FIELD_TOL = 2e-4   # m, m/s after the stated number of steps
FAST_DT_RTOL = 1e-4


@pytest.mark.parametrize("name,mk,nsteps", FAST_CASES, ids=[c[0] for c in FAST_CASES])
def test_fastmath_kernels_close_to_oracle(name, mk, nsteps):
    case = mk()
    case.param.fastmath = 1
    f, _, loop = make_gpu(case)
    o, _ = make_oracle(case)
    for s in range(nsteps):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert abs(dt - do) <= FAST_DT_RTOL * do, (s, dt, do)
    zs, h, u, v = f.get_state()
    for nm, a in (("h", h), ("u", u), ("v", v)):
        assert float(np.abs(interior(a).astype(np.float64) - interior(o.get(nm))).max()) <= FAST_FIELD_TOL, nm


@pytest.mark.parametrize("fast", [0, 1])
def test_fp32_eta_error_against_fp64_oracle(fast):
    """Both kernel variants in FP32 stay within 1e-3 m of the FP64 oracle on the
    wet/dry run-up case (2 s of simulated time, 128x128)."""
    case = cases.conical_island(128, 1)
    case.param.fastmath = fast
    f, mesh, loop = make_gpu(case)
    o, _ = make_oracle(case, use_double=True)
    loop.nextoutputtime = 2.0
    f.run(loop, endtime=2.0)
    o.set_loop(0.0, 2.0, o.init_loop(0.0, 2.0))
    while o.totaltime < 2.0:
        o.step(1)
    zs, h, u, v = f.get_state()
    err = float(np.abs(interior(zs).astype(np.float64) - interior(o.get("zs"))).max())
    assert err <= 1e-3, err


# ---------------------------------------------------------------- the benchmarked configurations

RUNUP_STEPS = 40
RUNUP_EXACT_TOL = 1e-5   # m, m/s: Manning's cbrtf rounds differently in glibc and CUDA
RUNUP_FP64_ETA_TOL = 1e-3  # m: FP32 surface against the FP64 oracle


@pytest.fixture(scope="module")
def runup_oracles():
    """The FP32 and FP64 oracles over the first RUNUP_STEPS steps of the benchmarked
    workload (1024x1024 run-up), with their dt sequences."""
    out = {}
    for dbl in (False, True):
        o, _ = make_oracle(cases.conical_island(1024, 1, dx=0.05), use_double=dbl)
        dts = [float(o.step(1)[0]) for _ in range(RUNUP_STEPS)]
        out[dbl] = (dts, {k: interior(o.get(k)).astype(np.float64) for k in ("zs", "h", "u", "v")})
    return out


@pytest.mark.parametrize("fast", [0, 1], ids=["exact", "fast"])
def test_runup1024_bench_workload_vs_oracle(fast, runup_oracles):
    """The workload bench.py times (1024x1024 cells, conical island, solitary wave,
    Manning n = 0.01), both kernel builds, against the FP32 oracle step by step and
    against the FP64 oracle at the end."""
    case = cases.conical_island(1024, 1, dx=0.05)
    case.param.fastmath = fast
    f, _, loop = make_gpu(case)
    dts, ref = runup_oracles[False]
    dt_rtol = FAST_DT_RTOL if fast else DT_RTOL
    for s in range(RUNUP_STEPS):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        assert abs(dt - dts[s]) <= dt_rtol * dts[s], (s, dt, dts[s])
    zs, h, u, v = f.get_state()
    tol = FAST_FIELD_TOL if fast else RUNUP_EXACT_TOL
    for nm, a in (("h", h), ("u", u), ("v", v)):
        assert float(np.abs(interior(a).astype(np.float64) - ref[nm]).max()) <= tol, nm
    _, ref64 = runup_oracles[True]
    eta_err = float(np.abs(interior(zs).astype(np.float64) - ref64["zs"]).max())
    assert eta_err <= RUNUP_FP64_ETA_TOL, eta_err


@pytest.mark.parametrize("fast", [0, 1], ids=["exact", "fast"])
def test_config1_hump256_full_run_vs_oracle(fast):
    """The plain-method configuration run in full: 256x256 cells, Gaussian hump on a
    flat bed 1 m deep, walls, Kurganov, no friction, 10 s simulated.  The exact build
    matches the oracle bit for bit at every step and in the fields; the fast build
    within the fast-math tolerances.  Volume is conserved either way."""
    case = cases.hump_walls(256, 2)
    case.param.fastmath = fast
    f, _, loop = make_gpu(case)
    o, _ = make_oracle(case)
    loop.nextoutputtime = 10.0
    o.set_loop(0.0, 10.0, loop.dtmax)
    v0 = f.volume()
    steps = 0
    while o.totaltime < 10.0:
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = float(o.step(1)[0])
        if fast:
            assert abs(dt - do) <= FAST_DT_RTOL * do, (steps, dt, do)
        else:
            assert dt == do, (steps, dt, do)
        steps += 1
    assert o.totaltime >= 10.0 and loop.totaltime == pytest.approx(o.totaltime, rel=1e-6 if fast else 0.0)
    zs, h, u, v = f.get_state()
    for nm, a in (("h", h), ("u", u), ("v", v)):
        d = float(np.abs(interior(a).astype(np.float64) - interior(o.get(nm))).max())
        assert d <= (FAST_FIELD_TOL if fast else 0.0), (nm, d)
    assert abs(f.volume() - v0) / v0 < 2e-6
