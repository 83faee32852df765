"""Gauges recorded on the device after every step (the reference's time-series
output nodes, pointoutputstep / storeTSout, src/Mainloop.cu:359-500): the series of
h, zs, u, v at the gauge cells and the step times equal the oracle's state after
each step, bit for bit, through the device loop and through single steps, alone
and in a pool."""
import numpy as np
import pytest

import cases
from bg_flood_b200.pool import ScenarioPool
from runners import make_gpu, make_oracle

pytestmark = pytest.mark.gpu

GAUGES = {"gauss48_e1_b3": [(0, 3, 5), (4, 15, 15), (8, 0, 7)],
          "hump64_e1": [(0, 0, 0), (5, 8, 8), (15, 15, 2), (10, 1, 14)],
          "hump64_e2": [(0, 0, 0), (5, 8, 8), (15, 15, 2), (10, 1, 14)]}
MK = {"gauss48_e1_b3": lambda: cases.gauss(48, 1, 3), "hump64_e1": lambda: cases.hump_walls(64, 1),
      "hump64_e2": lambda: cases.hump_walls(64, 2)}


def _oracle_series(name, nsteps):
    o, _ = make_oracle(MK[name]())
    t, v = [], []
    for _ in range(nsteps):
        o.step(1)
        t.append(o.totaltime)
        f = [o.get(k) for k in ("h", "zs", "u", "v")]
        v.append([[a[b, j + 1, i + 1] for a in f] for b, i, j in GAUGES[name]])
    return np.array(t), np.array(v)


@pytest.mark.parametrize("name", list(GAUGES))
def test_gauges_device_loop_match_oracle(name):
    nsteps = 30
    f, _, loop = make_gpu(MK[name]())
    f.set_gauges(GAUGES[name])
    assert f.run(loop, endtime=1e30, maxsteps=nsteps) == nsteps
    t, v, lost = f.read_gauges()
    ot, ov = _oracle_series(name, nsteps)
    assert lost == 0 and t.shape == (nsteps, len(GAUGES[name]))
    assert np.array_equal(t, np.repeat(ot[:, None], len(GAUGES[name]), 1))
    assert np.array_equal(v, ov.astype(np.float32).astype(np.float64))
    # nothing left after a read; single steps continue the series
    assert len(f.read_gauges()[0]) == 0


def test_gauges_single_steps_equal_device_loop():
    name = "gauss48_e1_b3"
    f1, _, l1 = make_gpu(MK[name]())
    f2, _, l2 = make_gpu(MK[name]())
    for f in (f1, f2):
        f.set_gauges(GAUGES[name])
    for _ in range(20):
        l1.totaltime += f1.flow_step(l1)
    f2.run(l2, endtime=1e30, maxsteps=20)
    t1, v1, _ = f1.read_gauges()
    t2, v2, _ = f2.read_gauges()
    assert np.array_equal(t1, t2) and np.array_equal(v1, v2) and len(t1) == 20


def test_gauges_in_a_pool_equal_alone():
    """Two scenarios with gauges in one pool, finishing at different steps: each
    scenario's series equals its series run alone; a retired scenario's unread
    samples go with its handle."""
    names = ["gauss48_e1_b3", "hump64_e1"]   # one engine per pool
    case0 = MK[names[0]]()
    pool = ScenarioPool(case0.param, 64, 4)
    slots, handles, steps = [], [], [24, 40]
    for name, n in zip(names, steps):
        f, _, loop = make_gpu(MK[name]())
        s = pool.admit(f, loop, 1e30, maxsteps=n)
        # pool gauges name the block by its index in the scenario's active order,
        # which on these uniform meshes is the block id
        pool.set_gauges(s, GAUGES[name])
        slots.append(s)
        handles.append(f)
    pool.run(8)
    first = pool.read_gauges(slots[1])
    assert pool.run(100) == 0
    for name, s, n in zip(names, slots, steps):
        t, v = pool.read_gauges(s)
        if s == slots[1]:
            t, v = np.concatenate([first[0], t]), np.concatenate([first[1], v])
        fa, _, la = make_gpu(MK[name]())
        fa.set_gauges(GAUGES[name])
        fa.run(la, endtime=1e30, maxsteps=n)
        ta, va, _ = fa.read_gauges()
        assert len(t) == n and np.array_equal(t, ta) and np.array_equal(v, va), name
    # samples recorded after a read and before retirement travel with the handle
    pool2 = ScenarioPool(case0.param, 64, 4)
    f, _, loop = make_gpu(MK[names[0]]())
    s = pool2.admit(f, loop, 1e30, maxsteps=12)
    pool2.set_gauges(s, [(0, 1, 1)])
    pool2.run(100)
    fr, _, _ = pool2.retire(s)
    t, v, _ = fr.read_gauges()
    assert len(t) == 12


def test_gauges_reject_cells_outside_the_mesh():
    from bg_flood_b200.flow import BGFError
    f, mesh, _ = make_gpu(cases.gauss(32, 1, 3))
    with pytest.raises(BGFError):
        f.set_gauges([(mesh.nblk, 0, 0)])
    with pytest.raises(BGFError):
        f.set_gauges([(0, 16, 0)])
