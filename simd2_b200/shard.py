"""Sharding of independent closure problems across ranks (one process per GPU).

The batched closure's graphs are independent, so a multi-GPU run needs no
exchange in the data path: each rank closes its own shard with one
persistent launch (simd2_b200.BatchedClosure) and only the per-graph step
counts and the timing are gathered.  Shards are balanced by
longest-processing-time on the work estimate n^3.
"""
from __future__ import annotations

import heapq


def assign_graphs(sizes, world: int):
    """Graph indices per rank: LPT over the cost n^3 (largest first onto the least-loaded rank).

    Deterministic for equal inputs, so every rank computes the same assignment
    without communication."""
    loads = [(0.0, r) for r in range(world)]
    heapq.heapify(loads)
    shards = [[] for _ in range(world)]
    for g in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        load, r = heapq.heappop(loads)
        shards[r].append(g)
        heapq.heappush(loads, (load + float(sizes[g]) ** 3, r))
    for s in shards:
        s.sort()
    return shards


def shard_imbalance(sizes, shards) -> float:
    """max / mean of the per-rank n^3 load (1.0 = perfect balance)."""
    loads = [sum(float(sizes[g]) ** 3 for g in s) for s in shards]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def gather_iters(local_graphs, local_iters, count: int, group=None):
    """All ranks' (graph, steps) pairs -> the full per-graph step list on every rank."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, list(zip(local_graphs, local_iters)), group=group)
    iters = [None] * count
    for part in parts:
        for g, it in part:
            iters[g] = it
    return iters


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The slowest rank's time (the bench reports max-over-ranks)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def run_batched_sharded(op: str, mats_by_graph, rank: int, world: int, max_iter: int = 500):
    """Closes this rank's shard of the graphs (dict or list index -> tensor) in
    one persistent launch; returns (graph indices, step counts)."""
    from . import BatchedClosure
    sizes = [m.shape[0] for m in mats_by_graph]
    mine = assign_graphs(sizes, world)[rank]
    plan = BatchedClosure(op, [mats_by_graph[g] for g in mine], max_iter=max_iter)
    plan.run()
    its, _ = plan.iters()
    plan.close()
    return mine, its
