"""The Kruskal oracle used for simd2_mst, checked against scipy's minimum
spanning tree (the total weight is unique even when weights tie) and
against the forest's defining properties."""
import numpy as np
import pytest
from scipy.sparse.csgraph import connected_components, minimum_spanning_tree

import oracle


@pytest.mark.parametrize("n,p,wmax,seed", [(50, 0.2, 5, 1), (200, 0.03, 10, 2), (120, 0.01, 100, 3)])
def test_oracle_mst_total_and_forest(n, p, wmax, seed):
    rng = np.random.default_rng(seed)
    x = np.where(rng.random((n, n)) < p, rng.integers(1, wmax + 1, (n, n)), np.inf).astype(np.float32)
    edges, weights = oracle.mst(x)
    s = np.minimum(x, x.T)
    dense = np.where(np.isfinite(s), s, 0)
    np.fill_diagonal(dense, 0)
    ref = minimum_spanning_tree(np.triu(dense)).toarray()
    assert weights.astype(np.float64).sum() == ref.sum()
    ncomp, _ = connected_components(dense > 0, directed=False)
    assert len(edges) == n - ncomp  # a spanning forest
    assert np.all(edges[:, 0] < edges[:, 1])
    assert np.all(s[edges[:, 0], edges[:, 1]] == weights)
