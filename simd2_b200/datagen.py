"""Seeded synthetic inputs for the srgemm / closure workloads.

The reference measures on generated graphs (``apps/data/graph_gen.h:33-81``,
``rgg_1d``/``rgg_1d_directed``, and the PaRMAT R-MAT generator) and on U[0,10)
point clouds for k-NN (``apps/pld/emulation/test.cpp:15-34``).  These
generators produce inputs of the same shapes and value distributions with
numpy's PCG64, so every run is reproducible from its seed.
"""
from __future__ import annotations

import numpy as np

MIN_ADD = ("min_plus", "min_mul", "min_max")
MAX_ADD = ("max_plus", "max_min", "max_mul")


def er_graph(n: int, p: float, seed: int, wmin: int = 1, wmax: int = 100, directed: bool = True,
             nonedge: float = np.inf, diag: float = 0.0) -> np.ndarray:
    """Erdos-Renyi adjacency matrix: integer weights U{wmin..wmax} stored as
    float32 on edges (probability p), ``nonedge`` elsewhere, ``diag`` on the
    diagonal (the APSP convention of apps/apsp/cuASR/apsp_cuASR.cu:77-93)."""
    rng = np.random.default_rng(seed)
    w = rng.integers(wmin, wmax + 1, size=(n, n)).astype(np.float32)
    e = rng.random((n, n)) < p
    if not directed:
        e = np.triu(e, 1)
        e = e | e.T
        w = np.triu(w, 1)
        w = w + w.T
    x = np.where(e, w, np.float32(nonedge)).astype(np.float32)
    np.fill_diagonal(x, np.float32(diag))
    return x


def closure_graph(op: str, n: int, p: float, seed: int) -> np.ndarray:
    """Graph for a closure under semiring ``op`` with the reference's
    conventions: APSP (min_plus) uses +inf non-edges and a 0 diagonal;
    maximum capacity (max_min) uses -inf for non-edges and the diagonal
    (apps/mcp/emulation/mcp_emulation.cu:134-141 uses -FLT_MAX)."""
    if op == "min_plus":
        return er_graph(n, p, seed)
    if op == "max_min":
        return er_graph(n, p, seed, nonedge=-np.inf, diag=-np.inf)
    if op == "max_plus":
        return er_graph(n, p, seed, nonedge=-np.inf, diag=-np.inf)
    if op == "min_max":
        return er_graph(n, p, seed, nonedge=np.inf, diag=0.0)
    raise ValueError(op)


def semiring_operands(op: str, m: int, n: int, k: int, seed: int, identity_frac: float = 0.2):
    """A (m x k), B (k x n), C (m x n) with the value distribution of the
    nine-semiring sweep: min/max semirings on integer-valued floats in
    [1,1000] with ``identity_frac`` entries set to the add-identity; the two
    *_mul semirings on U(0,1]; plus_mul / minus_square on N(0,1); or_and as
    uint8 Bernoulli(0.01)."""
    rng = np.random.default_rng(seed)
    if op == "or_and":
        a = (rng.random((m, k)) < 0.01).astype(np.uint8)
        b = (rng.random((k, n)) < 0.01).astype(np.uint8)
        c = (rng.random((m, n)) < 0.01).astype(np.uint8)
        return a, b, c
    if op in ("plus_mul", "minus_square"):
        return (rng.standard_normal((m, k), dtype=np.float32), rng.standard_normal((k, n), dtype=np.float32),
                rng.standard_normal((m, n), dtype=np.float32))
    if op in ("max_mul", "min_mul"):
        def u01(shape):
            return (1.0 - rng.random(shape, dtype=np.float32)).astype(np.float32)  # (0, 1]
        return u01((m, k)), u01((k, n)), u01((m, n))
    ident = np.float32(np.inf if op in MIN_ADD else -np.inf)

    def ints(shape):
        x = rng.integers(1, 1001, size=shape).astype(np.float32)
        x[rng.random(shape) < identity_frac] = ident
        return x
    return ints((m, k)), ints((k, n)), ints((m, n))


def batched_graphs(count: int, nmin: int, nmax: int, seed: int, op: str = "min_plus"):
    """``count`` graphs with N log-uniform in [nmin, nmax], edge probability
    U[0.01, 0.3], integer weights 1..100 (the batched-closure workload)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax + 1), size=count)).astype(np.int64)
    sizes = np.clip(sizes, nmin, nmax)
    probs = rng.uniform(0.01, 0.3, size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    return [closure_graph(op, int(n), float(p), int(s)) for n, p, s in zip(sizes, probs, seeds)]


def point_cloud(q: int, r: int, d: int, seed: int, dup_frac: float = 0.05, dup_offset: float = 1e-3):
    """Queries (q x d) and references (r x d) from N(0,1); a ``dup_frac``
    share of the queries is a reference point plus ``dup_offset`` noise,
    which makes near-duplicate pairs (the L2 cancellation band)."""
    rng = np.random.default_rng(seed)
    ref = rng.standard_normal((r, d), dtype=np.float32)
    query = rng.standard_normal((q, d), dtype=np.float32)
    ndup = int(round(q * dup_frac))
    if ndup:
        qi = rng.choice(q, size=ndup, replace=False)
        ri = rng.integers(0, r, size=ndup)
        query[qi] = ref[ri] + dup_offset * rng.standard_normal((ndup, d), dtype=np.float32)
    return query, ref


def rmat_graph(n: int, avg_degree: float, seed: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
               wmin: int = 1, wmax: int = 100) -> np.ndarray:
    """R-MAT directed graph (recursive quadrant choice with probabilities
    a, b, c, d = 1-a-b-c) with n*avg_degree edge draws, integer weights, +inf
    non-edges and a 0 diagonal; n must be a power of two."""
    rng = np.random.default_rng(seed)
    levels = int(np.log2(n))
    assert 1 << levels == n
    m = int(n * avg_degree)
    src = np.zeros(m, np.int64)
    dst = np.zeros(m, np.int64)
    for _ in range(levels):
        u = rng.random(m)
        right = (u >= a) & (u < a + b) | (u >= a + b + c)
        down = u >= a + b
        src = src * 2 + down
        dst = dst * 2 + right
    x = np.full((n, n), np.inf, np.float32)
    w = rng.integers(wmin, wmax + 1, size=m).astype(np.float32)
    # duplicate draws keep the smallest weight (a multigraph's shortest edge)
    order = np.argsort(-w, kind="stable")
    x[src[order], dst[order]] = w[order]
    np.fill_diagonal(x, 0.0)
    return x


def rmat_graph_device(n: int, avg_degree: float, seed: int, device, a: float = 0.57, b: float = 0.19,
                      c: float = 0.19, wmin: int = 1, wmax: int = 100):
    """The R-MAT graph of ``rmat_graph`` drawn on the GPU with torch's seeded
    generator (another random stream, so other graphs than the numpy
    version's): n * avg_degree edge draws, integer weights, duplicate draws
    keep the smallest weight, +inf non-edges, 0 diagonal.  Returns an n x n
    float32 CUDA tensor; n must be a power of two."""
    import torch
    levels = int(np.log2(n))
    assert 1 << levels == n
    m = int(n * avg_degree)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    src = torch.zeros(m, dtype=torch.int64, device=device)
    dst = torch.zeros(m, dtype=torch.int64, device=device)
    for _ in range(levels):
        u = torch.rand(m, generator=g, device=device)
        right = ((u >= a) & (u < a + b)) | (u >= a + b + c)
        down = u >= a + b
        src = src * 2 + down
        dst = dst * 2 + right
        del u, right, down
    w = torch.randint(wmin, wmax + 1, (m,), generator=g, device=device).float()
    x = torch.full((n * n,), float("inf"), dtype=torch.float32, device=device)
    x.scatter_reduce_(0, src * n + dst, w, reduce="amin")
    del src, dst, w
    x = x.view(n, n)
    x.fill_diagonal_(0.0)
    return x


def rmat_mixed_set(count: int = 64, seed: int = 5):
    """The mixed-density R-MAT workload: (n, average degree, seed) for
    ``count`` graphs, n cycling through 4096, 8192, 16384 and the degree
    log-uniform in [4, 4096]."""
    rng = np.random.default_rng(seed)
    degs = np.exp(rng.uniform(np.log(4.0), np.log(4096.0), size=count))
    seeds = rng.integers(0, 2**31 - 1, size=count)
    return [((4096, 8192, 16384)[i % 3], float(round(float(d), 2)), int(s)) for i, (d, s) in enumerate(zip(degs, seeds))]
