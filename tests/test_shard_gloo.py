"""Multi-rank logic on CPU (gloo, world sizes 2 and 3): sharding, gathering,
max-over-ranks, and the row-panel closure's exchange loop (with the oracle
as the per-rank panel step)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from simd2_b200 import datagen
from simd2_b200.shard import (assign_graphs, closure_rowpanel, gather_iters, max_over_ranks, panel_bounds,
                              shard_imbalance)


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shards = assign_graphs(sizes, world)
        mine = shards[rank]
        fake_iters = [3 + (g % 5) for g in mine]  # stand-in for a GPU shard's step counts
        iters = gather_iters(mine, fake_iters, len(sizes))
        slowest = max_over_ranks(1.0 + rank)
        q.put((rank, mine, iters, slowest))
    finally:
        dist.destroy_process_group()


def test_assignment_is_a_balanced_partition():
    sizes = [int(n) for n in np.exp(np.random.default_rng(0).uniform(np.log(32), np.log(1025), 4096))]
    for world in (1, 2, 4, 8):
        shards = assign_graphs(sizes, world)
        flat = sorted(g for s in shards for g in s)
        assert flat == list(range(len(sizes)))
        assert shard_imbalance(sizes, shards) < 1.02
        assert assign_graphs(sizes, world) == shards  # deterministic


def test_two_rank_gather_and_max():
    sizes = [g.shape[0] for g in datagen.batched_graphs(64, 32, 256, seed=1)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (_, mine0, iters0, slow0), (_, mine1, iters1, slow1) = out
    assert sorted(mine0 + mine1) == list(range(len(sizes)))
    assert iters0 == iters1 == [3 + (g % 5) for g in range(len(sizes))]
    assert slow0 == slow1 == 2.0


# --- one large closure split by row panels -------------------------------

def _oracle_panel_step(op, panel, full, out, changed, conv):
    """The panel step on the CPU with the oracle (the GPU step is
    simd2_closure_panel_step): out = panel (+) panel (x) full, change flag."""
    import oracle
    p = panel.numpy()
    new = oracle.srgemm(op, p, full.numpy(), p, do_epilogue=True, threads=1)
    out.copy_(torch.from_numpy(new))
    if not np.array_equal(new.view(np.uint8), np.ascontiguousarray(p).view(np.uint8)):
        changed.fill_(1)


def _rowpanel_worker(rank, world, port, op, x, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = x.shape[0]
        P, bounds = panel_bounds(n, world)
        start, stop = bounds[rank]
        block = torch.zeros((P, n), dtype=torch.from_numpy(x).dtype)
        block[: stop - start] = torch.from_numpy(x[start:stop])
        it = closure_rowpanel(op, block, n, step=_oracle_panel_step)
        q.put((rank, start, stop, block[: stop - start].numpy().copy(), it))
    finally:
        dist.destroy_process_group()


def _run_rowpanel(op, x, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rowpanel_worker, args=(r, world, port, op, x, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out, key=lambda t: t[0])


def test_panel_bounds_cover_rows_once():
    for n in (0, 1, 7, 128, 1000, 4097):
        for world in (1, 2, 3, 4, 8):
            P, b = panel_bounds(n, world)
            assert len(b) == world and b[0][0] == 0 and b[-1][1] == n
            assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            assert all(0 <= stop - start <= P for start, stop in b)


def test_rowpanel_closure_two_ranks_min_plus():
    import oracle
    x = datagen.er_graph(96, 0.04, seed=3)
    want, it_want = oracle.closure("min_plus", x)
    parts = _run_rowpanel("min_plus", x, 2)
    got = np.concatenate([p[3] for p in parts])
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert all(p[4] == it_want for p in parts)


def test_rowpanel_closure_three_ranks_uneven_or_and():
    """n = 70 over 3 ranks: blocks of 24, 24 and 22 rows (padding in the last)."""
    import oracle
    rng = np.random.default_rng(4)
    x = (rng.random((70, 70)) < 0.03).astype(np.uint8)
    np.fill_diagonal(x, 1)
    want, it_want = oracle.closure("or_and", x)
    parts = _run_rowpanel("or_and", x, 3)
    assert [p[2] - p[1] for p in parts] == [24, 24, 22]
    got = np.concatenate([p[3] for p in parts])
    assert np.array_equal(got, want)
    assert all(p[4] == it_want for p in parts)
