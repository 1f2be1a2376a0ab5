"""Replica plumbing on CPU: the cost partition and the max-over-ranks timing
reduction with two gloo ranks (the collective bench.py uses for N > 1)."""
import os
import socket

import pytest

from mettleq_b200.replicas import partition_by_cost


def test_partition_covers_every_unit_once_and_balances():
    costs = [2 ** n for n in (10, 24, 13, 20, 24, 11, 18, 22, 15, 12)]
    parts = partition_by_cost(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= max(costs) + min(loads)
    assert partition_by_cost(costs, 3) == parts  # deterministic
    assert partition_by_cost([], 2) == [[], []]
    with pytest.raises(ValueError):
        partition_by_cost(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from mettleq_b200.replicas import max_over_ranks, partition_by_cost
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = max_over_ranks(0.5 + rank, dist)
        mine = partition_by_cost([5, 1, 4, 2, 3, 8], world)[rank]
        q.put((rank, t, mine))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [t for _, t, _ in got] == [1.5, 1.5]
    assert sorted(i for _, _, m in got for i in m) == list(range(6))
