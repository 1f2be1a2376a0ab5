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


def test_request_assignment_by_work():
    from mettleq_b200.serving import assign_by_work, poisson_requests
    reqs = poisson_requests(60, seed=3, depth_range=(1, 3))
    parts = assign_by_work(reqs, 4)
    assert sorted(i for p in parts for i in p) == list(range(60))
    assert assign_by_work(reqs, 4) == parts
    loads = [sum(reqs[i].work for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(r.work for r in reqs)
    # online: a request's device depends only on earlier arrivals
    first = assign_by_work(reqs[:30], 4)
    for d in range(4):
        assert [i for i in parts[d] if i < 30] == first[d]
    assert assign_by_work(reqs, 1) == [list(range(60))]
    with pytest.raises(ValueError):
        assign_by_work(reqs, 0)


def _share_rank(rank, world, port, q):
    """One rank of a replicated batch and request stream: its share by the
    same deterministic rules, results gathered to every rank."""
    import datetime
    import torch.distributed as dist
    from mettleq_b200.batch import hea_batch
    from mettleq_b200.replicas import gather_objects, partition_by_cost
    from mettleq_b200.serving import assign_by_work, poisson_requests
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ns, ds, _ = hea_batch(64, seed=2)
        mine_b = partition_by_cost([d << n for n, d in zip(ns, ds)], world)[rank]
        reqs = poisson_requests(40, seed=5, depth_range=(1, 3))
        mine_s = assign_by_work(reqs, world)[rank]
        # stand-ins for per-request results: latency = rank + position
        res = [(i, rank + 0.001 * i) for i in mine_s]
        q.put((rank, gather_objects(mine_b, dist), gather_objects(res, dist)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_a_batch_and_a_request_stream():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_share_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=60) for _ in range(2)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # every rank sees the same gathered lists, covering every unit once
    assert got[0][1] == got[1][1] and got[0][2] == got[1][2]
    assert sorted(i for part in got[0][1] for i in part) == list(range(64))
    ids = sorted(i for part in got[0][2] for i, _ in part)
    assert ids == list(range(40))
    assert all(lat == pytest.approx(r + 0.001 * i) for r, part in enumerate(got[0][2]) for i, lat in part)


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
