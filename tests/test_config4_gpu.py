"""The dense-contraction workloads at full size, checked through properties
that do not need the full CPU result:
  * or_and transitive closure, N = 16384, edge probability 2/N (INT8 tensor
    cores): sampled rows equal BFS reachability from those vertices;
  * k-NN, Q = 16384 queries x R = 65536 references x D = 128, k = 16, with 5 %
    near-duplicate queries: sampled queries against the FP64 oracle;
  * plus_mul 8192^3 on N(0,1) (BF16 hi/lo): sampled rows inside the FP64 bound.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import breadth_first_order
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu


def test_orand_closure_16384(cuda):
    n = 16384
    rng = np.random.default_rng(44)
    m = int(2 * n)  # expected edges at p = 2/N
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    X = torch.zeros((n, n), dtype=torch.uint8, device=cuda)
    X[torch.from_numpy(src).to(cuda), torch.from_numpy(dst).to(cuda)] = 1
    X.fill_diagonal_(1)
    it = s2.closure("or_and", X)
    assert 2 <= it <= 40
    adj = sp.csr_matrix((np.ones(m, np.int8), (src, dst)), shape=(n, n))
    for v in rng.choice(n, size=64, replace=False):
        reach = np.zeros(n, np.uint8)
        reach[breadth_first_order(adj, int(v), directed=True, return_predecessors=False)] = 1
        np.testing.assert_array_equal(X[int(v)].cpu().numpy(), reach, err_msg=f"row {v}")
    assert s2.device_status() == 0


def test_knn_16384_x_65536(cuda):
    """256 sampled queries (all near-duplicate queries among them checked on
    their own) against the FP64 oracle: every returned squared distance
    within the stated bound of the returned reference's true distance, the
    neighbour sets equal up to near-ties (>= 99.8 % of indices in place), and
    the near-duplicate queries' nearest distance to FP32 relative accuracy
    (the exact recompute of the cancellation band)."""
    q, r = datagen.point_cloud(16384, 65536, 128, seed=4, dup_frac=0.05)
    Q, R = torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda)
    dist, idx = s2.knn(Q, R, 16)
    torch.cuda.synchronize()
    dist, idx = dist.cpu().numpy(), idx.cpu().numpy()
    sample = np.random.default_rng(0).choice(16384, size=256, replace=False)
    want_d, want_i, want_sq = oracle.knn(q[sample], r, 16)
    match = (idx[sample] == want_i).mean()
    assert match >= 0.998, match
    qs = q[sample].astype(np.float64)
    ri = r[idx[sample]].astype(np.float64)
    true_sq = ((qs[:, None, :] - ri) ** 2).sum(-1)
    nq = (qs ** 2).sum(1)[:, None]
    nr = (ri ** 2).sum(-1)
    bound = (4 * 2.0 ** -16 + 2 * 128 * 2.0 ** -24) * 2 * (nq + nr)
    got_sq = dist[sample].astype(np.float64) ** 2
    assert np.all(np.abs(got_sq - true_sq) <= bound + 1e-6 * true_sq)
    assert np.all(np.abs(np.sort(true_sq, 1) - want_sq) <= bound)
    near = np.sqrt(want_sq[:, 0]) < 0.1
    assert near.sum() >= 5
    rel = np.abs(dist[sample][near, 0].astype(np.float64) - np.sqrt(want_sq[near, 0])) / np.sqrt(want_sq[near, 0])
    assert rel.max() <= 1e-5, rel.max()


def test_plus_mul_8192(cuda):
    n = 8192
    a, b, _ = datagen.semiring_operands("plus_mul", n, n, 1, seed=5)
    rng = np.random.default_rng(6)
    a = rng.standard_normal((n, n), dtype=np.float32)
    b = rng.standard_normal((n, n), dtype=np.float32)
    D = s2.srgemm("plus_mul", torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda))
    rows = rng.choice(n, size=8, replace=False)
    got = D[torch.from_numpy(rows).to(cuda)].cpu().numpy().astype(np.float64)
    want = oracle.srgemm_f64("plus_mul", a[rows], b)
    bound = (4 * 2.0 ** -16 + 2 * n * 2.0 ** -24) * (np.abs(a[rows]).astype(np.float64) @ np.abs(b))
    assert np.all(np.abs(got - want) <= bound)


def test_orand_closure_delta_steps_match_plain_steps(cuda):
    """The or_and closure squares X in place and, from its second dense step,
    skips every 256 x 256 tile whose tile row and tile column did not change in
    the step before.  The whole closed matrix and the step count must equal a
    loop of plain or_and srgemm steps X <- X | X & X (fresh output each step,
    no skipping) run until X stops changing."""
    n = 12288
    rng = np.random.default_rng(46)
    m = 2 * n
    src = torch.from_numpy(rng.integers(0, n, m)).to(cuda)
    dst = torch.from_numpy(rng.integers(0, n, m)).to(cuda)
    X0 = torch.zeros((n, n), dtype=torch.uint8, device=cuda)
    X0[src, dst] = 1
    X0.fill_diagonal_(1)
    X = X0.clone()
    it = s2.closure("or_and", X)
    Y = X0.clone()
    steps = 0
    while True:
        Z = s2.srgemm("or_and", Y, Y, Y, do_epilogue=True)
        steps += 1
        if torch.equal(Z, Y):
            break
        Y = Z
    assert it == steps
    assert torch.equal(X, Y)
    assert s2.device_status() == 0
