"""Closure with a predecessor matrix on the GPU (simd2_closure_pred) against
the oracle, bit-exact in X and P, and against the closed-form results of the
reference's Floyd-Warshall tests at their size (1000 vertices)."""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

from test_pred_oracle import dicircle_edges, expected, fw_input, k1_edges, kn_edges

pytestmark = pytest.mark.gpu

OPS = ["min_plus", "max_plus", "max_min", "max_mul", "min_mul", "min_max"]


def graph(op, n, seed):
    if op in ("max_mul", "min_mul"):
        rng = np.random.default_rng(seed)
        x = np.where(rng.random((n, n)) < 0.05, rng.uniform(0.05, 1.0, (n, n)),
                     0.0 if op == "max_mul" else np.inf).astype(np.float32)
        np.fill_diagonal(x, 1.0)
        return x
    x = datagen.closure_graph(op, n, 0.04, seed)
    if op == "max_plus":
        x = np.where(np.triu(np.ones((n, n), bool), 1), x, -np.inf).astype(np.float32)
    return x


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("n", [1, 65, 203])
def test_closure_pred_matches_oracle(cuda, op, n):
    x = graph(op, n, seed=n)
    want_x, want_p, want_it = oracle.closure_pred(op, x)
    X = torch.from_numpy(x).to(cuda)
    it, P = s2.closure_pred(op, X)
    assert it == want_it
    assert np.array_equal(X.cpu().numpy().view(np.uint32), want_x.view(np.uint32))
    np.testing.assert_array_equal(P.cpu().numpy(), want_p)


TIE_IDENT = {"min_plus": np.inf, "max_plus": -np.inf, "max_min": -np.inf, "min_max": np.inf}


@pytest.mark.parametrize("op", list(TIE_IDENT))
@pytest.mark.parametrize("n", [300, 512])
def test_closure_pred_ties(cuda, op, n):
    """Small integer weights: most (i, j) have many k attaining the best
    product, within one 32-wide k-tile and across k-tiles, so the witness must
    be the lowest such k exactly as in the sequential accumulation."""
    rng = np.random.default_rng(n + len(op))
    x = np.where(rng.random((n, n)) < 0.2, rng.integers(1, 4, (n, n)), TIE_IDENT[op]).astype(np.float32)
    if op == "max_plus":  # a DAG: no positive cycles
        x = np.where(np.triu(np.ones((n, n), bool), 1), x, -np.inf).astype(np.float32)
    want_x, want_p, want_it = oracle.closure_pred(op, x)
    X = torch.from_numpy(x).to(cuda)
    it, P = s2.closure_pred(op, X)
    assert it == want_it
    assert np.array_equal(X.cpu().numpy().view(np.uint32), want_x.view(np.uint32))
    np.testing.assert_array_equal(P.cpu().numpy(), want_p)


@pytest.mark.parametrize("family,edges", [("k0", lambda n: []), ("k1", k1_edges), ("kn", kn_edges),
                                          ("dicircle", dicircle_edges)])
def test_fw_families_1000(cuda, family, edges):
    n = 1000
    X = torch.from_numpy(fw_input(n, edges(n))).to(cuda)
    _, P = s2.closure_pred("min_plus", X)
    g, p = expected(n, family)
    Xh = X.cpu().numpy()
    np.testing.assert_array_equal(np.where(np.isinf(Xh), -1, Xh).astype(np.int64), g)
    np.testing.assert_array_equal(P.cpu().numpy(), p)


def test_pitched_buffers_and_given_p(cuda):
    """Row pitches above n, and a caller-initialised P (init_pred = 0)."""
    n = 150
    x = graph("min_plus", n, seed=3)
    _, p0, _ = oracle.closure_pred("min_plus", x, max_iter=0)
    want_x, want_p, want_it = oracle.closure_pred("min_plus", x)
    Xb = torch.full((n, n + 13), 7.0, device=cuda)
    Pb = torch.full((n, n + 5), 99, dtype=torch.int32, device=cuda)
    Xb[:, :n] = torch.from_numpy(x).to(cuda)
    Pb[:, :n] = torch.from_numpy(p0).to(cuda)
    it, _ = s2.closure_pred("min_plus", Xb[:, :n], Pb[:, :n])
    assert it == want_it
    assert np.array_equal(Xb[:, :n].cpu().numpy().view(np.uint32), want_x.view(np.uint32))
    np.testing.assert_array_equal(Pb[:, :n].cpu().numpy(), want_p)
    assert torch.all(Xb[:, n:] == 7.0) and torch.all(Pb[:, n:] == 99)


def test_recorded_paths_are_shortest(cuda):
    n = 400
    x = graph("min_plus", n, seed=9)
    X = torch.from_numpy(x).to(cuda)
    _, P = s2.closure_pred("min_plus", X)
    Xh, Ph = X.cpu().numpy(), P.cpu().numpy()
    rng = np.random.default_rng(0)
    for i, j in rng.integers(0, n, (300, 2)):
        pth = s2.path(Ph, int(i), int(j))
        if np.isinf(Xh[i, j]):
            assert pth == []
            continue
        assert sum(float(x[u, v]) for u, v in zip(pth, pth[1:])) == Xh[i, j]


def test_closure_pred_rejects_sum_semirings(cuda):
    X = torch.zeros((8, 8), device=cuda)
    with pytest.raises(s2.Simd2Error):
        s2.closure_pred("plus_mul", X)
