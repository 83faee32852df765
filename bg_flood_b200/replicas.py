"""Multi-GPU use of the flow step: independent replicas, one process per GPU.

The path has no exchange step between independent scenarios, so N GPUs run N
replicas (or disjoint shares of a scenario list) with no data-path collective;
the process group only provides the barrier and the max-over-ranks timing of a
measurement."""
from __future__ import annotations


def scenario_share(n: int, rank: int, world: int) -> list[int]:
    """Indices of the scenarios rank `rank` runs out of n, round-robin so that the
    ranks' shares differ by at most one scenario."""
    return list(range(rank, n, world))


def replica_throughput(units_per_rank: float, local_ms: float, dist=None, device=None):
    """Whole-job throughput of N replicas: units processed by all ranks divided by
    the slowest rank's time (max over ranks).  Returns (units per second, max ms)."""
    world = 1
    tmax = float(local_ms)
    if dist is not None and dist.is_available() and dist.is_initialized():
        import torch
        world = dist.get_world_size()
        t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tmax = float(t.item())
    return world * units_per_rank / (tmax / 1e3), tmax
