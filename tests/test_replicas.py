"""The N>1 path on CPU: two gloo ranks shard the 64-seed batch and reduce their timings."""
import os
import socket

import pytest

from slime_b200 import replicas, workloads


def test_replica_seeds_distinct_and_signed():
    base = workloads.full_world_scan().seed
    seeds = [replicas.replica_seed(base, r) for r in range(8)]
    assert seeds[0] == base and len(set(seeds)) == 8
    assert all(-(1 << 63) <= s < (1 << 63) for s in seeds)


def test_shard_requests_partition_and_balance():
    searches = workloads.batch_searches()
    for world in (1, 2, 4, 8):
        shards = [replicas.shard_requests(searches, r, world) for r in range(world)]
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(searches)))
        loads = [sum(searches[i].centres for i in s) for s in shards]
        biggest = max(q.centres for q in searches)
        assert max(loads) - min(loads) <= biggest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        searches = workloads.batch_searches()
        mine = replicas.shard_requests(searches, rank, world)
        centres = sum(searches[i].centres for i in mine)
        fake_time = 1.0 + rank  # stands in for this rank's measured batch time
        (t_max,), (c_sum, n_sum) = replicas.reduce_max_sum(dist, [fake_time], [centres, len(mine)])
        out.put((rank, t_max, c_sum, n_sum, mine))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_shard_the_batch_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = [out.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    searches = workloads.batch_searches()
    total = sum(q.centres for q in searches)
    for rank, t_max, c_sum, n_sum, mine in got:
        assert t_max == 2.0 and c_sum == total and n_sum == len(searches)
    assert sorted(i for *_, mine in got for i in mine) == list(range(len(searches)))
