"""Minimum spanning forest from the min_max closure (simd2_mst) against
Kruskal over all edges in (weight, u, v) order: the same edges in the same
order, the same total -- with many equal weights, disconnected graphs and
asymmetric input."""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2

pytestmark = pytest.mark.gpu


def graph(n, p, wmax, seed, symmetric=True):
    rng = np.random.default_rng(seed)
    w = rng.integers(1, wmax + 1, (n, n)).astype(np.float32)
    e = rng.random((n, n)) < p
    x = np.where(e, w, np.inf).astype(np.float32)
    if symmetric:
        x = np.minimum(x, x.T)
    return x


@pytest.mark.parametrize("n,p,wmax,sym", [(2, 1.0, 5, True), (3, 0.0, 5, True), (64, 0.1, 10, True),
                                          (300, 0.05, 10, True), (301, 0.02, 1000, False), (500, 0.003, 7, True)])
def test_mst_matches_kruskal(cuda, n, p, wmax, sym):
    x = graph(n, p, wmax, seed=n + wmax, symmetric=sym)
    edges, weights, total, it = s2.mst(torch.from_numpy(x).to(cuda))
    want_e, want_w = oracle.mst(x)
    np.testing.assert_array_equal(edges, want_e)
    np.testing.assert_array_equal(weights, want_w)
    assert total == pytest.approx(float(want_w.astype(np.float64).sum()), rel=0, abs=0)


def test_mst_trivial_sizes(cuda):
    for n in (0, 1):
        e, w, total, it = s2.mst(torch.zeros((n, n), device=cuda))
        assert len(e) == 0 and total == 0.0
