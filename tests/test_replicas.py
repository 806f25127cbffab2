"""Host logic of the multi-GPU replica mode: job placement and the max-over-ranks timing
reduction, with two gloo ranks on the CPU (one process per rank, as under torchrun)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from tsne_h2pack._replicas import job_cost, max_over_ranks, shard


def test_shard_partitions_and_balances():
    costs = [job_cost(n) for n in (2000, 50000, 3000, 49000, 10000, 7000, 2500, 30000)]
    for world in (1, 2, 3, 8):
        parts = shard(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        if world == 2:
            assert max(loads) / min(loads) < 1.2
    assert shard(costs, 2) == shard(list(costs), 2)
    assert shard([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        shard(costs, 0)


def test_max_over_ranks_without_group():
    assert max_over_ranks([1.5, 2.0]) == [1.5, 2.0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        costs = [job_cost(n) for n in (5000, 200000, 12000, 80000, 6000)]
        mine = shard(costs, world)[rank]
        # each rank "times" its share: the slowest rank's value must come back on every rank
        local = [float(sum(costs[i] for i in mine)), float(rank)]
        q.put((rank, mine, max_over_ranks(local)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    costs = [job_cost(n) for n in (5000, 200000, 12000, 80000, 6000)]
    expect = shard(costs, world)
    assert [r[1] for r in res] == expect
    assert sorted(i for r in res for i in r[1]) == list(range(5))
    loads = [sum(costs[i] for i in p) for p in expect]
    for _, _, m in res:
        assert m == [max(loads), float(world - 1)]
