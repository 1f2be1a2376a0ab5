"""Multi-GPU plumbing for independent replicas (no data-path collective).

A 30-qubit state fits one B200 and batched / served circuits are independent,
so several GPUs run replicas: each rank (one process per GPU) takes its share
of the units (``partition_by_cost`` for a batch, ``serving.assign_by_work``
for a request stream), and the only collectives are the timing reduction
(the slowest rank's time defines the job's time) and the gathering of
per-rank results.  One state larger than a GPU is sharded instead
(``mettleq_b200.sharded``).
"""
from __future__ import annotations

from typing import List, Sequence


def partition_by_cost(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time assignment of units to ``world`` ranks: units
    in decreasing cost, each to the currently least-loaded rank (ties to the
    lowest rank).  Deterministic, so every rank computes the same plan."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    for p in parts:
        p.sort()
    return parts


def gather_objects(obj, dist=None) -> list:
    """Every rank's ``obj`` in rank order, on every rank (a pickled
    all-gather; for per-rank results such as latency lists and counters)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def max_over_ranks(seconds: float, dist=None, device: str = "cpu") -> float:
    """The largest ``seconds`` over all ranks (every rank calls it, in the same
    order as its other collectives)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(seconds)
    import torch
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
