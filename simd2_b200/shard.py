"""Multi-GPU closures, one process per GPU.

Independent graphs (the batched closure): no exchange in the data path.
Each rank closes its own shard with one persistent launch
(simd2_b200.BatchedClosure) and only the per-graph step counts and the timing
are gathered.  Shards are balanced by longest-processing-time on the work
estimate n^3.

One large closure (closure_rowpanel): each rank owns a row panel of X.  A
squaring step needs all of X as the right operand, so the step is one
all-gather of the panels, the rank's panel step on its own GPU
(simd2_closure_panel_step), and one all-reduce (MAX) of the change flag --
the reference's single-GPU loop (apps/apsp/cuASR/apsp_cuASR.cu:37-54) with
X's rows distributed.
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


def panel_bounds(n: int, world: int):
    """(P, [(start, stop) per rank]): every rank holds a block of P = ceil(n / world)
    rows, of which rows [start, stop) of X are its own (the last ranks may own
    fewer, or none).  Equal block heights let the ranks all-gather fixed-size
    blocks, and the first n rows of the gathered buffer are then X."""
    P = -(-n // world) if n else 0
    return P, [(min(n, r * P), min(n, (r + 1) * P)) for r in range(world)]


def closure_rowpanel(op: str, block, n: int, group=None, max_iter: int = 500, conv: str = "exact", step=None):
    """Repeated squaring X <- X (+) X (x) X of an n x n matrix split by rows across the ranks of ``group``.

    ``block`` is this rank's P x n block (``panel_bounds``); its first
    stop - start rows are the rank's rows of X and receive the closed rows.
    Returns the step count (every rank returns the same).  Raises
    NotConverged when X still changed after ``max_iter`` steps.

    ``step(op, panel, full, out, changed, conv)`` computes one panel step;
    the default is simd2_b200.closure_panel_step on the block's GPU.
    """
    import torch
    import torch.distributed as dist
    from . import NotConverged, closure_panel_step
    step = step or closure_panel_step
    if max_iter <= 0:
        return 0
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if dist_on else 1
    rank = dist.get_rank(group) if dist_on else 0
    P, bounds = panel_bounds(n, world)
    start, stop = bounds[rank]
    rows = stop - start
    if block.shape != (P, n):
        raise ValueError(f"rank {rank}: block must be {P} x {n}, got {tuple(block.shape)}")
    cur, nxt = block, torch.empty_like(block)
    full = torch.empty((world * P, n), dtype=block.dtype, device=block.device) if world > 1 else None
    changed = torch.zeros(1, dtype=torch.int32, device=block.device)
    it, more = 0, n > 0
    while more and it < max_iter:
        it += 1
        if world > 1:
            dist.all_gather_into_tensor(full, cur, group=group)
            X = full[:n]
        else:
            X = cur
        changed.zero_()
        if rows:
            step(op, cur[:rows], X, nxt[:rows], changed, conv)
        if world > 1:
            dist.all_reduce(changed, op=dist.ReduceOp.MAX, group=group)
        more = bool(changed.item())
        cur, nxt = nxt, cur
    if cur is not block and rows:
        block[:rows].copy_(cur[:rows])
    if more:
        raise NotConverged(6, f"closure_rowpanel({op}): still changing after {max_iter} steps")
    return it
