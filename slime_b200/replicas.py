"""Multi-GPU helpers: the search shards by independent requests, with no data-path collective.

One process per GPU. A single search runs on one GPU (its areas are independent of every other
rank's); a batch of requests is split across ranks by expected work (centres), each rank runs
its share with the batched kernel, and only the timing is reduced (max over ranks, on the host's
process group). Nothing here touches a GPU, so the logic is tested with gloo ranks on CPU.
"""
from __future__ import annotations

GOLDEN = 0x9E3779B97F4A7C15


def replica_seed(base_seed: int, rank: int) -> int:
    """World seed of replica `rank` (rank 0 keeps the base seed), as a signed 64-bit value."""
    s = (base_seed + rank * GOLDEN) % (1 << 64)
    return s - (1 << 64) if s >> 63 else s


def shard_requests(searches, rank: int, world: int):
    """Indices of the requests rank `rank` runs: longest-first greedy balance of the centres each
    request scans (deterministic; every request lands on exactly one rank)."""
    if world <= 1:
        return list(range(len(searches)))
    load = [0] * world
    owner = [0] * len(searches)
    for i in sorted(range(len(searches)), key=lambda i: (-searches[i].centres, i)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += searches[i].centres
    return [i for i in range(len(searches)) if owner[i] == rank]


def reduce_max_sum(dist, values_max, values_sum, device=None):
    """(max over ranks of values_max, sum over ranks of values_sum) through torch.distributed."""
    import torch
    t_max = torch.tensor(values_max, dtype=torch.float64, device=device)
    t_sum = torch.tensor(values_sum, dtype=torch.float64, device=device)
    dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    dist.all_reduce(t_sum, op=dist.ReduceOp.SUM)
    return t_max.tolist(), t_sum.tolist()
