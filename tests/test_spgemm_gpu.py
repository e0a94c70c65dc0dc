"""Semiring SpGEMM and the sparse closure against the oracle (the dense
host_srgemm contract with absent entries = the add identity): values bit for
bit, structure = the Boolean product's pattern (plus C's)."""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu

OPS = ["min_plus", "max_plus", "max_min", "min_max", "plus_mul"]


def sparse_dense(op, rows, cols, density, rng):
    """Dense array with the add identity where nothing is stored."""
    ident = s2.SPARSE_IDENTITY[op]
    if op == "plus_mul":
        vals = rng.standard_normal((rows, cols)).astype(np.float32)
    else:
        vals = rng.integers(1, 101, (rows, cols)).astype(np.float32)
    keep = rng.random((rows, cols)) < density
    return np.where(keep, vals, np.float32(ident)).astype(np.float32), keep


def to_csr(x, op, dev):
    return s2.csr_from_dense(torch.from_numpy(x).to(dev), op)


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("shape", [(1, 1, 1), (37, 61, 50), (300, 400, 200), (130, 70, 257), (20, 20000, 30)])
@pytest.mark.parametrize("with_c", [False, True])
def test_spgemm_matches_dense_oracle(cuda, op, shape, with_c):
    M, N, K = shape
    rng = np.random.default_rng(M * 7 + N + K + with_c)
    a, pa = sparse_dense(op, M, K, 0.05, rng)
    b, pb = sparse_dense(op, K, N, 0.05, rng)
    c, pc = sparse_dense(op, M, N, 0.03, rng)
    A, B = to_csr(a, op, cuda), to_csr(b, op, cuda)
    C = to_csr(c, op, cuda) if with_c else None
    D = s2.spgemm(op, A, B, N, C=C)
    got = s2.csr_to_dense(D, N, op).cpu().numpy()
    want = oracle.srgemm(op, a, b, c if with_c else None, do_epilogue=with_c)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    pattern = (pa.astype(np.int64) @ pb.astype(np.int64)) > 0
    if with_c:
        pattern |= pc
    dp, dj, _ = (t.cpu().numpy() for t in D)
    got_pattern = np.zeros((M, N), bool)
    for i in range(M):
        row = dj[dp[i]:dp[i + 1]]
        assert np.all(np.diff(row) > 0)  # sorted, no duplicates
        got_pattern[i, row] = True
    assert np.array_equal(got_pattern, pattern)


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("density", [0.002, 0.05])
def test_spgemm_sparse_and_dense_results(cuda, op, density):
    """4096 columns (shared-memory accumulators) with results on both sides of
    the 1/32 average row density at which the min/max fill switches between
    its bitmap form (0.002: ~0.2 % dense) and its keys-only form (0.05:
    ~70 % dense); with C, against the dense oracle bit for bit."""
    M, N, K = 64, 4096, 512
    rng = np.random.default_rng(int(density * 1000) + len(op))
    a, _ = sparse_dense(op, M, K, density, rng)
    b, _ = sparse_dense(op, K, N, density, rng)
    c, _ = sparse_dense(op, M, N, density, rng)
    D = s2.spgemm(op, to_csr(a, op, cuda), to_csr(b, op, cuda), N, C=to_csr(c, op, cuda))
    nnz = D[1].numel()
    assert (nnz <= M * N // 32) == (density < 0.01)
    got = s2.csr_to_dense(D, N, op).cpu().numpy()
    want = oracle.srgemm(op, a, b, c, do_epilogue=True)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("n_cols", [300, 17000])
def test_spgemm_dense_ties(cuda, op, n_cols):
    """Dense-ish operands with values in {1, 2}: many products meet on every
    output column from different k (the min/max fill folds them from
    different warps without ordering), with accumulators in shared memory
    (300 columns) and in the global scratch (17000 columns)."""
    rng = np.random.default_rng(n_cols)
    ident = np.float32(s2.SPARSE_IDENTITY[op])
    a = np.where(rng.random((48, 200)) < 0.6, rng.integers(1, 3, (48, 200)), ident).astype(np.float32)
    b = np.where(rng.random((200, n_cols)) < 0.6, rng.integers(1, 3, (200, n_cols)), ident).astype(np.float32)
    c = np.where(rng.random((48, n_cols)) < 0.3, rng.integers(1, 3, (48, n_cols)), ident).astype(np.float32)
    D = s2.spgemm(op, to_csr(a, op, cuda), to_csr(b, op, cuda), n_cols, C=to_csr(c, op, cuda))
    got = s2.csr_to_dense(D, n_cols, op).cpu().numpy()
    want = oracle.srgemm(op, a, b, c, do_epilogue=True)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_spgemm_empty_rows_and_matrices(cuda):
    op = "min_plus"
    a = np.full((5, 4), np.inf, np.float32)
    a[2, 1] = 3
    b = np.full((4, 6), np.inf, np.float32)
    b[1, 5] = 4
    D = s2.spgemm(op, to_csr(a, op, cuda), to_csr(b, op, cuda), 6)
    dp, dj, dv = (t.cpu().numpy() for t in D)
    assert list(dp) == [0, 0, 0, 1, 1, 1] and list(dj) == [5] and list(dv) == [7.0]
    z = np.full((3, 3), np.inf, np.float32)
    D = s2.spgemm(op, to_csr(z, op, cuda), to_csr(z, op, cuda), 3)
    assert D[1].numel() == 0 and list(D[0].cpu().numpy()) == [0, 0, 0, 0]


def test_spgemm_rejects_malformed_csr(cuda):
    op = "min_plus"
    rp = torch.tensor([0, 2, 3], dtype=torch.int32, device=cuda)
    good = (rp, torch.tensor([0, 2, 1], dtype=torch.int32, device=cuda), torch.ones(3, device=cuda))
    unsorted = (rp, torch.tensor([2, 0, 1], dtype=torch.int32, device=cuda), torch.ones(3, device=cuda))
    outside = (rp, torch.tensor([0, 7, 1], dtype=torch.int32, device=cuda), torch.ones(3, device=cuda))
    bad_end = (torch.tensor([0, 2, 5], dtype=torch.int32, device=cuda), good[1], good[2])
    B = s2.csr_from_dense(torch.ones((3, 3), device=cuda), op)
    s2.spgemm(op, good, B, 3)
    for bad in (unsorted, outside, bad_end):
        with pytest.raises(s2.Simd2Error):
            s2.spgemm(op, bad, B, 3)
    with pytest.raises(s2.Simd2Error):
        s2.spgemm("max_mul", good, B, 3)


def chains(op, n, length, rng):
    """Disjoint directed paths of `length` vertices: the closure stays sparse."""
    ident = s2.SPARSE_IDENTITY[op]
    x = np.full((n, n), ident, np.float32)
    if op == "min_plus" or op == "min_max":
        np.fill_diagonal(x, 0)
    for s0 in range(0, n - length + 1, length):
        for v in range(s0, s0 + length - 1):
            x[v, v + 1] = rng.integers(1, 101)
    return x


@pytest.mark.parametrize("op", ["min_plus", "max_min", "min_max"])
@pytest.mark.parametrize("case", ["switch", "sparse_only", "dense_start"])
def test_closure_sparse_matches_oracle(cuda, op, case):
    """The three regimes of the hybrid closure: fill-in past density 1/32
    (sparse steps, then the dense closure), convergence while still sparse,
    and an input already denser than the threshold."""
    n = 400
    if case == "switch":
        x = datagen.closure_graph(op, n, 0.004, seed=13)
    elif case == "sparse_only":
        n = 2000
        x = chains(op, n, 6, np.random.default_rng(3))
    else:
        x = datagen.closure_graph(op, n, 0.05, seed=14)
    ident = s2.SPARSE_IDENTITY[op]
    X = to_csr(x, op, cuda)
    closed, it = s2.closure_sparse(op, X)
    want, it_want = oracle.closure(op, x)
    got = s2.csr_to_dense(closed, n, op).cpu().numpy()
    # the dense closure keeps the diagonal's identity entries as stored values; compare densified
    assert it == it_want
    assert np.array_equal(got.view(np.uint32), np.where(want == ident, np.float32(ident), want).view(np.uint32))


def test_closure_sparse_capacity(cuda):
    op = "min_plus"
    n = 200
    x = datagen.closure_graph(op, n, 0.01, seed=2)
    X = to_csr(x, op, cuda)
    nnz0 = X[1].numel()
    with pytest.raises(s2.Simd2Error) as e:
        s2.closure_sparse(op, X, capacity=nnz0)
    assert e.value.status == 8
