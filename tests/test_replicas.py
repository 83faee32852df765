"""Multi-GPU replicas on CPU: two gloo ranks, the max-over-ranks throughput and the
scenario shares (no data-path collective exists on this path)."""
import os

import pytest
import torch.multiprocessing as mp

from bg_flood_b200.replicas import replica_throughput, scenario_share


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        local_ms = 10.0 * (rank + 1)      # rank 1 is the slowest
        val, tmax = replica_throughput(1000.0, local_ms, dist, device="cpu")
        share = scenario_share(11, rank, world)
        q.put((rank, val, tmax, share))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, val, tmax, share in res:
        assert tmax == 20.0                      # the slowest rank's time on every rank
        assert val == pytest.approx(2 * 1000.0 / 0.020)
    shares = [s for _, _, _, s in res]
    assert sorted(shares[0] + shares[1]) == list(range(11)) and not set(shares[0]) & set(shares[1])


def test_single_process_throughput():
    val, tmax = replica_throughput(500.0, 5.0)
    assert tmax == 5.0 and val == pytest.approx(500.0 / 0.005)
