"""Split precision (FP32 deviations from per-block datums) against the FP64 build
on deep-water cases: the surface error stays below 1e-3 m where plain FP32 does
not, a deep lake at rest stays at rest, and shallow cases keep the accuracy of
plain FP32."""
import numpy as np
import pytest

import cases
from runners import interior, make_gpu

pytestmark = pytest.mark.gpu


def run_to(case, endtime, mode):
    """mode: 'fp32', 'split' or 'fp64'; returns (zs, hu) interior arrays in double."""
    case.param.doubleprecision = 1 if mode == "fp64" else 0
    case.param.splitprecision = 1 if mode == "split" else 0
    case.nextoutputtime = endtime
    f, mesh, loop = make_gpu(case)
    f.run(loop, endtime=endtime)
    assert abs(loop.totaltime - endtime) < 1e-6  # the FP32 builds take their last dt in FP32
    zs, h, u, v = f.get_state()
    zs, h, u = (interior(a).astype(np.float64) for a in (zs, h, u))
    return zs, h * u


@pytest.mark.parametrize("k", [3, 7])
def test_tsunami_surface_error_below_1mm(k):
    T = 300.0
    ref = run_to(cases.ensemble_member(k, 2024, 64, 512), T, "fp64")
    sp = run_to(cases.ensemble_member(k, 2024, 64, 512), T, "split")
    f32 = run_to(cases.ensemble_member(k, 2024, 64, 512), T, "fp32")
    e_split = float(np.abs(sp[0] - ref[0]).max())
    e_f32 = float(np.abs(f32[0] - ref[0]).max())
    assert e_split <= 1e-3, e_split
    assert e_split < 0.5 * e_f32, (e_split, e_f32)


def test_deep_lake_at_rest():
    """A flat surface over the 4000 m basin with its 3800 m ridge stays flat: split
    precision keeps the drift at the resolution of the deviations of the ridge's
    blocks (whose beds span the whole depth range), far below plain FP32."""
    def lake():
        case = cases.ensemble_member(3, 2024, 64, 512)
        case.h = np.maximum(0.0 - case.zb, 0.0).astype(np.float32)   # flat surface at 0
        return case
    zs_s, hu_s = run_to(lake(), 200.0, "split")
    zs_f, hu_f = run_to(lake(), 200.0, "fp32")
    e_s, e_f = float(np.abs(zs_s).max()), float(np.abs(zs_f).max())
    assert e_s <= 2.5e-4 and e_s < 0.25 * e_f, (e_s, e_f)


def test_shallow_cases_keep_fp32_accuracy():
    T = 2.0
    for mk in (lambda: cases.dam_break(48, 1), lambda: cases.conical_island(64, 2)):
        ref = run_to(mk(), T, "fp64")
        sp = run_to(mk(), T, "split")
        f32 = run_to(mk(), T, "fp32")
        e_split = float(np.abs(sp[0] - ref[0]).max())
        e_f32 = float(np.abs(f32[0] - ref[0]).max())
        assert e_split <= max(2.0 * e_f32, 1e-5), (e_split, e_f32)


def oracle_to(case, endtime, use_double):
    """The CPU oracle (FP64 or FP32 restatement of FlowCPU) to `endtime`; (zs, hu)."""
    from runners import make_oracle
    case.nextoutputtime = endtime
    o, _ = make_oracle(case, use_double=use_double)
    while o.totaltime < endtime:
        o.step(1)
    assert abs(o.totaltime - endtime) < 1e-6  # the FP32 build accumulates its time in FP32 steps
    zs, h, u = (interior(o.get(k)) for k in ("zs", "h", "u"))
    return zs, h * u


@pytest.mark.parametrize("fastmath", [0, 1])
def test_tsunami_error_vs_fp64_oracle(fastmath):
    """Against the FP64 oracle: the split-precision surface stays within 1e-3 m after
    300 s, while the reference's own FP32 arithmetic (the oracle's FP32 build) does not
    get as close."""
    T = 300.0
    mk = lambda: cases.ensemble_member(3, 2024, 64, 512)
    ref = oracle_to(mk(), T, True)
    f32 = oracle_to(mk(), T, False)
    c = mk()
    c.param.fastmath = fastmath
    sp = run_to(c, T, "split")
    e_split = float(np.abs(sp[0] - ref[0]).max())
    e_f32 = float(np.abs(f32[0] - ref[0]).max())
    assert e_split <= 1e-3, e_split
    assert e_split < 0.5 * e_f32, (e_split, e_f32)


@pytest.mark.parametrize("fastmath", [0, 1])
def test_rain_member_error_is_the_fp32_reference_error(fastmath):
    """Rain on fractal terrain (dry start, 300 s): FP32 evaluation of the reference's
    algorithm moves water into different pits than FP64 does, by centimetres -- the
    oracle's FP32 build differs from its FP64 build as much as the split-precision
    GPU build does.  The bound: the GPU error is at most the reference-FP32 error
    plus 1e-3 m, for the surface and for the unit discharge (plus 1e-2 m2/s)."""
    T = 300.0
    mk = lambda: cases.ensemble_member(1, 2024, 64, 1024)
    ref = oracle_to(mk(), T, True)
    f32 = oracle_to(mk(), T, False)
    c = mk()
    c.param.fastmath = fastmath
    sp = run_to(c, T, "split")
    e_split, q_split = (float(np.abs(sp[i] - ref[i]).max()) for i in (0, 1))
    e_f32, q_f32 = (float(np.abs(f32[i] - ref[i]).max()) for i in (0, 1))
    assert e_f32 > 1e-3  # the FP32 reference itself is outside 1 mm here
    assert e_split <= e_f32 + 1e-3, (e_split, e_f32)
    assert q_split <= q_f32 + 1e-2, (q_split, q_f32)
