"""Multi-rank logic on CPU (gloo, world size 2): sharding, gathering, max-over-ranks."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from simd2_b200 import datagen
from simd2_b200.shard import assign_graphs, gather_iters, max_over_ranks, shard_imbalance


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
