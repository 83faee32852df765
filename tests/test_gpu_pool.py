"""Batched pool: scenarios of different sizes, forcings and boundaries advanced
together give bit for bit the results they give alone (same kernels, own dt per
scenario), including scenarios admitted while others are running."""
import numpy as np
import pytest

import cases
from bg_flood_b200.pool import ScenarioPool
from runners import interior, make_gpu

pytestmark = pytest.mark.gpu

MIX = [
    lambda: cases.gauss(48, 1, 3),
    lambda: cases.dam_break(48, 1),
    lambda: cases.conical_island(64, 1),
    lambda: cases.rain_on_terrain(48, 1),
    lambda: cases.hump_walls(32, 1),
]
ENDTIME = 1e30
BUDGET = [40, 55, 70, 85, 100]   # steps per scenario: they finish at different pool steps


def alone(mk, maxsteps):
    f, mesh, loop = make_gpu(mk())
    n = f.run(loop, endtime=ENDTIME, maxsteps=maxsteps)
    return f.get_state(), loop, n


def test_pool_results_equal_alone():
    ref = [alone(mk, n) for mk, n in zip(MIX, BUDGET)]
    case0 = MIX[0]()
    pool = ScenarioPool(case0.param, 4096, 8)
    slots = []
    for mk, n in zip(MIX, BUDGET):
        f, mesh, loop = make_gpu(mk())
        slots.append(pool.admit(f, loop, ENDTIME, maxsteps=n))
    left = pool.run(100000)
    assert left == 0
    for s, (st, loop_a, n_a) in zip(slots, ref):
        f, loop, n = pool.retire(s)
        assert n == n_a and loop.totaltime == loop_a.totaltime and loop.dt == loop_a.dt
        for a, b in zip(f.get_state()[1:], st[1:]):
            assert np.array_equal(interior(a), interior(b))


def test_pool_admission_while_running():
    """Continuous batching: B joins after A has run 30 steps; C replaces A when A ends."""
    mkA, mkB, mkC = MIX[1], MIX[2], MIX[4]
    budget = {"A": 80, "B": 120, "C": 60}
    ref = {k: alone(mk, budget[k]) for k, mk in (("A", mkA), ("B", mkB), ("C", mkC))}
    pool = ScenarioPool(mkA().param, 1200, 2)
    fA, _, lA = make_gpu(mkA())
    sA = pool.admit(fA, lA, ENDTIME, maxsteps=budget["A"])
    pool.run(30)
    fB, _, lB = make_gpu(mkB())
    sB = pool.admit(fB, lB, ENDTIME, maxsteps=budget["B"])
    fC, _, lC = make_gpu(mkC())
    assert pool.try_admit(fC, lC, ENDTIME, maxsteps=budget["C"]) is None  # two scenario slots only
    names = {sA: "A", sB: "B"}
    pending = [("C", fC, lC)]
    done = {}
    while len(done) < 3:
        pool.run(64)
        for s in list(names):
            loop, status, n = pool.query(s)
            if status:
                f, loop, n = pool.retire(s)
                done[names.pop(s)] = (f.get_state(), loop, n)
                if pending:
                    k, f2, l2 = pending.pop()
                    names[pool.admit(f2, l2, ENDTIME, maxsteps=budget[k])] = k
    for k, (st, loop, n) in done.items():
        st_a, loop_a, n_a = ref[k]
        assert n == n_a and loop.totaltime == loop_a.totaltime, k
        for a, b in zip(st[1:], st_a[1:]):
            assert np.array_equal(interior(a), interior(b)), k


def test_pool_tracks_maximum_depth():
    mk = MIX[1]
    pool = ScenarioPool(mk().param, 512, 1, track_hmax=True)
    f, mesh, loop = make_gpu(mk())
    h0 = interior(f.get_state()[1])
    s = pool.admit(f, loop, ENDTIME, maxsteps=60)
    pool.run(100000)
    h, hmax = pool.depth(s, mesh.nblk, with_max=True)
    assert np.all(hmax >= h) and np.all(hmax >= h0)
    assert float((hmax - h).max()) > 0.0


def test_pool_with_multilevel_scenarios():
    """Adapted (2- and 3-level) and single-level scenarios in one pool: the pool takes
    the multi-level chain, and every result still equals the one run alone."""
    import os
    from runners import make_gpu_amr
    golden = os.path.join(os.path.dirname(__file__), "golden")

    def amr(name, mk):
        g = np.load(os.path.join(golden, f"{name}.npz"))
        return lambda: make_gpu_amr(mk(), (g["level"], g["nbr"], g["xo"], g["yo"]))

    def single(mk):
        def b():
            f, mesh, loop = make_gpu(mk())
            return f, loop
        return b

    members = [
        (amr("amrhump64_e1_l1", lambda: cases.amr_hump(64, 1, 1, 0.3)), 45),
        (amr("amrdam64_e1_l2", lambda: cases.amr_dambreak(64, 1, 2)), 30),
        (single(lambda: cases.dam_break(48, 1)), 50),
        (single(lambda: cases.gauss(32, 1, 0)), 35),
    ]
    ref = []
    for build, n in members:
        f, loop = build()
        assert f.run(loop, endtime=ENDTIME, maxsteps=n) == n
        ref.append((f.get_state(), loop))
    pool = ScenarioPool(cases.dam_break(48, 1).param, 4096, 4)
    slots = []
    for build, n in members:
        f, loop = build()
        slots.append(pool.admit(f, loop, ENDTIME, maxsteps=n))
    assert pool.run(100000) == 0
    for s, (st, loop_a), (_, n) in zip(slots, ref, members):
        f, loop, nn = pool.retire(s)
        assert nn == n and loop.totaltime == loop_a.totaltime and loop.dt == loop_a.dt
        for a, b in zip(f.get_state()[1:], st[1:]):
            assert np.array_equal(interior(a), interior(b))


@pytest.mark.parametrize("prepare", [False, True], ids=["rebuild_at_run", "prepare_behind_run"])
def test_async_run_and_batched_finish(prepare):
    """Chunks enqueued with run_async while the scenarios that finished in the last
    chunk are retired with finish (fields gathered on the pool's copy stream): every
    scenario's final depth, maximum depth, time and step count equal its run alone,
    a later admission reuses freed slots, and a scenario still running cannot be
    finished.  With prepare, the tables after each retirement are rebuilt while the
    chunk runs (bgf_pool_prepare) instead of by the next run_async."""
    from bg_flood_b200.flow import BGFError
    ref = [alone(mk, n) for mk, n in zip(MIX, BUDGET)]
    case0 = MIX[0]()
    pool = ScenarioPool(case0.param, 4096, 8, track_hmax=True)
    built = [make_gpu(mk()) for mk in MIX]
    slots = {pool.admit(f, loop, ENDTIME, maxsteps=n): k for k, ((f, mesh, loop), n) in enumerate(zip(built, BUDGET))}
    # a running scenario is refused
    pool.run(4)
    with pytest.raises(BGFError):
        pool.finish([next(iter(slots))], [built[slots[next(iter(slots))]][1].nblk])
    got, finished = {}, []
    while slots:
        running = len(slots) > len(finished)
        if running:
            pool.run_async(16)
        if finished:
            res = pool.finish(finished, [built[slots[s]][1].nblk for s in finished], with_max=True)
            for s, (f, h, hmax, loop, n, status) in zip(finished, res):
                got[slots.pop(s)] = (h, hmax, loop, n, status)
            finished = []
        if not running:
            continue
        if prepare:
            pool.prepare()
        pool.wait()
        for s in slots:
            _, status, _ = pool.query(s)
            if status != 0:
                finished.append(s)
    for k, (st, loop_a, n_a) in enumerate(ref):
        h, hmax, loop, n, status = got[k]
        assert status == 1 and n == n_a and loop.totaltime == loop_a.totaltime, k
        nblk = built[k][1].nblk
        assert np.array_equal(h, interior(st[1])[:nblk]), k
        assert (hmax >= h).all(), k
    # the freed slots take a new scenario, which again matches its run alone
    (st, loop_a, n_a) = alone(MIX[1], 30)
    f, mesh, loop = make_gpu(MIX[1]())
    s = pool.admit(f, loop, ENDTIME, maxsteps=30)
    assert pool.run(1000) == 0
    (_, h, _, loop_p, n_p, _), = pool.finish([s], [mesh.nblk])
    assert n_p == n_a and np.array_equal(h, interior(st[1])[: mesh.nblk])
    pool.close()


def test_admission_prepared_behind_a_running_chunk():
    """Scenarios admitted while a chunk is in flight, with the next chunk's tables
    built at once (bgf_pool_prepare, uploads queued behind the chunk): they join
    the next chunk, which run_async launches without a rebuild, and every scenario
    ends as it does alone; a second prepare with nothing pending changes nothing."""
    ref = [alone(mk, n) for mk, n in zip(MIX[:3], [60, 45, 50])]
    case0 = MIX[0]()
    pool = ScenarioPool(case0.param, 4096, 8, track_hmax=True)
    built = [make_gpu(mk()) for mk in MIX[:3]]
    s0 = pool.admit(built[0][0], built[0][2], ENDTIME, maxsteps=60)
    pool.run_async(16)
    s1 = pool.admit(built[1][0], built[1][2], ENDTIME, maxsteps=45)   # queued behind the chunk
    s2 = pool.admit(built[2][0], built[2][2], ENDTIME, maxsteps=50)
    pool.prepare()
    pool.prepare()
    assert pool.wait() >= 1
    _, st1, n1 = pool.query(s1)
    assert st1 == 0 and n1 == 0   # not yet stepped
    while True:
        pool.run_async(16)
        pool.prepare()            # nothing pending: no effect
        if pool.wait() == 0:
            break
    for s, (st, loop_a, n_a), (f, mesh, _) in zip((s0, s1, s2), ref, built):
        loop, status, n = pool.query(s)
        assert n == n_a and loop.totaltime == loop_a.totaltime
        assert np.array_equal(pool.depth(s, mesh.nblk), interior(st[1])[: mesh.nblk])
    pool.close()


def test_three_prepares_behind_one_chunk():
    """Three admissions while one chunk is in flight, each followed by
    bgf_pool_prepare: three table rebuilds queued behind the same chunk, so the third
    reuses the staging area of the first before any wait (its copies must have run
    first).  Every scenario still ends as it does alone."""
    steps = [60, 45, 50, 35]
    ref = [alone(mk, n) for mk, n in zip(MIX[:4], steps)]
    pool = ScenarioPool(MIX[0]().param, 4096, 8)
    built = [make_gpu(mk()) for mk in MIX[:4]]
    slots = [pool.admit(built[0][0], built[0][2], ENDTIME, maxsteps=steps[0])]
    pool.run_async(16)
    for k in (1, 2, 3):
        slots.append(pool.admit(built[k][0], built[k][2], ENDTIME, maxsteps=steps[k]))
        pool.prepare()
    while True:
        if pool.wait() == 0:
            break
        pool.run_async(16)
    for s, (st, loop_a, n_a), (f, mesh, _) in zip(slots, ref, built):
        loop, status, n = pool.query(s)
        assert n == n_a and loop.totaltime == loop_a.totaltime
        assert np.array_equal(pool.depth(s, mesh.nblk), interior(st[1])[: mesh.nblk])
    pool.close()


def test_admission_queued_behind_a_running_chunk():
    """Scenarios admitted (with gauges) while a chunk is in flight join the next
    chunk and end as they do alone; the running scenario is unaffected."""
    ref = [alone(mk, n) for mk, n in zip(MIX[:3], [60, 45, 50])]
    case0 = MIX[0]()
    pool = ScenarioPool(case0.param, 4096, 8, track_hmax=True)
    built = [make_gpu(mk()) for mk in MIX[:3]]
    s0 = pool.admit(built[0][0], built[0][2], ENDTIME, maxsteps=60)
    pool.run_async(16)
    s1 = pool.admit(built[1][0], built[1][2], ENDTIME, maxsteps=45)   # queued behind the chunk
    s2 = pool.admit(built[2][0], built[2][2], ENDTIME, maxsteps=50)
    pool.set_gauges(s2, [(0, 3, 4)])
    assert pool.wait() >= 1
    _, st1, n1 = pool.query(s1)
    assert st1 == 0 and n1 == 0   # not yet stepped
    assert pool.run(1000) == 0
    for s, (st, loop_a, n_a), (f, mesh, _) in zip((s0, s1, s2), ref, built):
        loop, status, n = pool.query(s)
        assert n == n_a and loop.totaltime == loop_a.totaltime
        assert np.array_equal(pool.depth(s, mesh.nblk), interior(st[1])[: mesh.nblk])
    t, v = pool.read_gauges(s2)
    assert len(t) == 50
    pool.close()
