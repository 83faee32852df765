"""Serving loop: a stream of scenarios of different sizes run through the pool
under an HBM budget smaller than the whole stream; every result equals the one
the scenario gives alone (same steps, same final state) and the maximum-depth map
bounds the depth."""
import numpy as np
import pytest

import cases
from bg_flood_b200.serve import FloodServer, Request, bytes_per_block_slot, serve_sequential
from runners import make_gpu

pytestmark = pytest.mark.gpu


def _requests(n, steps=60):
    reqs = []
    for k in range(n):
        case = cases.ensemble_member(k, seed=11, min_blocks=4, max_blocks=64)

        def build(case=case):
            f, mesh, loop = make_gpu(case)
            return f, loop
        nblk = (case.nx // 16) * (case.ny // 16)
        reqs.append(Request(k, arrival=0.002 * k, nblk=nblk, build=build, maxsteps=steps + 7 * k,
                            gauges=[(0, 0), (nblk - 1, 255)]))
    return reqs


def test_served_results_equal_alone():
    reqs = _requests(10)
    budget = bytes_per_block_slot() * 150   # fewer slots than the whole stream needs
    srv = FloodServer(cases.ensemble_member(0, 11).param, budget, max_scenarios=4, chunk_steps=16)
    res = srv.serve(reqs, realtime=True)
    assert len(res) == len(reqs)
    for r, q in zip(res, reqs):
        f, loop = q.build()
        act = f.get_blocks()[0]
        f.set_gauges([(int(act[b]), c % 16, c // 16) for b, c in q.gauges])
        n = f.run(loop, endtime=q.endtime, maxsteps=q.maxsteps)
        h = f.get_state()[1][: q.nblk, 1:17, 1:17]
        assert r.nsteps == n and r.totaltime == loop.totaltime
        assert np.array_equal(r.h, h)
        assert np.all(r.hmax >= r.h)
        assert r.time_to_solution > 0
        # gauges recorded on the device after every step, alone and served
        t, v, lost = f.read_gauges()
        assert lost == 0 and len(t) == n == len(r.gauge_series)
        assert [s[0] for s in r.gauge_series] == t[:, 0].tolist()
        assert np.array_equal(np.array([s[1] for s in r.gauge_series]), v[:, :, 0])
    seq = serve_sequential(reqs, realtime=False)
    assert [s.nsteps for s in seq] == [r.nsteps for r in res]
