"""A non-finite value in the state stops its scenario with BGF_ENAN (status 5)
instead of running on silently: the single step, the device loop, the
multi-level chain and a pool, where the other scenarios continue unaffected."""
import os

import numpy as np
import pytest

import cases
from bg_flood_b200.flow import BGFError
from bg_flood_b200.pool import ScenarioPool
from runners import interior, make_gpu, make_gpu_amr

pytestmark = pytest.mark.gpu
BGF_ENAN = 5


def poisoned(case, value=np.nan):
    n = case.h.shape[0]
    case.u[n // 2, n // 3] = value
    return case


@pytest.mark.parametrize("value", [np.nan, np.inf])
def test_flow_step_reports_nonfinite_state(value):
    f, mesh, loop = make_gpu(poisoned(cases.dam_break(64, 1), value))
    with pytest.raises(BGFError) as e:
        f.flow_step(loop)
    assert e.value.status == BGF_ENAN


def test_run_stops_on_nonfinite_state():
    f, mesh, loop = make_gpu(poisoned(cases.gauss(64, 2, 3)))
    with pytest.raises(BGFError) as e:
        f.run(loop, endtime=1e30, maxsteps=50)
    assert e.value.status == BGF_ENAN
    assert loop.totaltime == 0.0


def test_multilevel_chain_stops_on_nonfinite_state():
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "amrdam64_e1_l2.npz"))
    f, loop = make_gpu_amr(cases.amr_dambreak(64, 1, 2), (g["level"], g["nbr"], g["xo"], g["yo"]))
    zs, h, u, v = f.get_state()
    wet = np.argwhere(interior(h) > 0)[0]
    v[wet[0], wet[1] + 1, wet[2] + 1] = np.nan
    f.set_state(h, u, v)
    with pytest.raises(BGFError) as e:
        f.run(loop, endtime=1e30, maxsteps=20)
    assert e.value.status == BGF_ENAN


def test_finite_states_unchanged():
    # the check changes nothing for a finite state: same dt sequence as before
    f, _, loop = make_gpu(cases.dam_break(64, 1))
    dts = [f.flow_step(loop) for _ in range(5)]
    assert all(d > 0 for d in dts)


def test_pool_isolates_nonfinite_scenario():
    good = lambda: cases.dam_break(48, 1)
    ref, _, lref = make_gpu(good())
    ref.run(lref, endtime=1e30, maxsteps=40)
    pool = ScenarioPool(good().param, 256, 2)
    fg, _, lg = make_gpu(good())
    fb, _, lb = make_gpu(poisoned(good()))
    sg = pool.admit(fg, lg, 1e30, maxsteps=40)
    sb = pool.admit(fb, lb, 1e30, maxsteps=40)
    assert pool.run(1000) == 0
    assert pool.query(sb)[1] == 3
    assert pool.query(sg)[1] == 1
    f, loop, n = pool.retire(sg)
    assert n == 40 and loop.totaltime == lref.totaltime
    for a, b in zip(f.get_state()[1:], ref.get_state()[1:]):
        assert np.array_equal(interior(a), interior(b))
