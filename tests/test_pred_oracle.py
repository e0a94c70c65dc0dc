"""The predecessor-matrix oracle against the closed-form results of the
reference's Floyd-Warshall tests (apps/maxrp/baseline/test/test_apsp/
test_basic.py with helpers.py: empty graph, K0, K1 pairs, complete graph Kn,
directed circle -- every shortest path unique, so the predecessors are
determined), and path validity on random graphs."""
import numpy as np
import pytest

import oracle
from simd2_b200 import datagen


def fw_input(n, edges):
    """The baselines' input convention: +inf without an edge, 0 on the diagonal."""
    x = np.full((n, n), np.inf, np.float32)
    for u, v, w in edges:
        x[u, v] = w
    np.fill_diagonal(x, 0)
    return x


def k1_edges(n):
    return [(2 * i, 2 * i + 1, 1) for i in range(n // 2)] + [(2 * i + 1, 2 * i, 1) for i in range(n // 2)]


def kn_edges(n):
    return [(i, j, 1) for i in range(n) for j in range(n) if i != j]


def dicircle_edges(n):
    return [(i, i + 1, 1) for i in range(n - 1)] + [(n - 1, 0, 1)]


def expected(n, family):
    """(distances with -1 for no path, predecessors) as the reference's tests state them."""
    g = np.full((n, n), -1, np.int64)
    p = np.full((n, n), -1, np.int64)
    np.fill_diagonal(g, 0)
    if family == "k1":
        for i in range(n // 2):
            g[2 * i, 2 * i + 1] = g[2 * i + 1, 2 * i] = 1
            p[2 * i, 2 * i + 1], p[2 * i + 1, 2 * i] = 2 * i, 2 * i + 1
    elif family == "kn":
        g[:] = 1
        np.fill_diagonal(g, 0)
        p[:] = np.arange(n)[:, None]
        np.fill_diagonal(p, -1)
    elif family == "dicircle":
        i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        g = (j - i) % n
        p = (j - 1) % n
        np.fill_diagonal(p, -1)
    return g, p


@pytest.mark.parametrize("family,edges", [("k0", lambda n: []), ("k1", k1_edges), ("kn", kn_edges),
                                          ("dicircle", dicircle_edges)])
def test_fw_families(family, edges):
    n = 60
    X, P, _ = oracle.closure_pred("min_plus", fw_input(n, edges(n)))
    g, p = expected(n, family)
    got_g = np.where(np.isinf(X), -1, X).astype(np.int64)
    np.testing.assert_array_equal(got_g, g)
    np.testing.assert_array_equal(P, p)


def test_empty_graph():
    X, P, it = oracle.closure_pred("min_plus", np.zeros((0, 0), np.float32))
    assert X.shape == (0, 0) and P.shape == (0, 0)


@pytest.mark.parametrize("op", ["min_plus", "max_min", "min_max", "max_plus"])
def test_paths_realise_the_closure(op):
    """Every recorded path exists in the graph and its (x)-product is the
    closed value (integer weights: exact)."""
    n = 70
    x = datagen.closure_graph(op, n, 0.06, seed=5)
    if op == "max_plus":  # keep it acyclic so the longest paths are finite
        x = np.where(np.triu(np.ones((n, n), bool), 1), x, -np.inf).astype(np.float32)
    X, P, _ = oracle.closure_pred(op, x)
    ident = np.inf if op in ("min_plus", "min_max") else -np.inf
    mul = {"min_plus": lambda a, b: a + b, "max_plus": lambda a, b: a + b, "max_min": min, "min_max": max}[op]
    for i in range(n):
        for j in range(n):
            if i == j:
                continue
            pth = oracle.path(P, i, j)
            if X[i, j] == ident:
                assert pth == [] and P[i, j] == -1
                continue
            assert pth[0] == i and pth[-1] == j
            acc = x[pth[0], pth[1]]
            for u, v in zip(pth[1:], pth[2:]):
                assert x[u, v] != ident
                acc = mul(acc, x[u, v])
            assert acc == X[i, j], (i, j, pth)
