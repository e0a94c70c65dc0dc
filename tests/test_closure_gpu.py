"""GPU closure (repeated squaring) against the oracle's closure loop."""
import os

import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def bits(x):
    return np.ascontiguousarray(x).view(np.uint32)


def gpu_closure(op, x, dev, **kw):
    X = torch.from_numpy(x.copy()).to(dev)
    it = s2.closure(op, X, **kw)
    return X.cpu().numpy(), it


def test_apsp_er_512(cuda):
    """Plain APSP on a directed ER graph, N=512, p=0.05, weights 1..100."""
    x = datagen.er_graph(512, 0.05, seed=1)
    want, it_want = oracle.closure("min_plus", x)
    got, it = gpu_closure("min_plus", x, cuda)
    assert it == it_want
    np.testing.assert_array_equal(bits(got), bits(want))


@pytest.mark.parametrize("op", ["min_plus", "max_min"])
def test_closure_golden(cuda, op):
    g = np.load(os.path.join(GOLDEN, f"closure_{op}.npz"))
    got, it = gpu_closure(op, g["X0"], cuda)
    assert it == int(g["iters"])
    np.testing.assert_array_equal(bits(got), bits(g["X"]))


@pytest.mark.parametrize("op", ["min_plus", "max_min", "max_plus", "min_max"])
@pytest.mark.parametrize("n", [1, 31, 130, 257])
def test_closure_ops_sizes(cuda, op, n):
    x = datagen.closure_graph(op, n, 0.05, seed=n)
    if op == "max_plus":  # max_plus closure only terminates on a DAG
        x = np.where(np.triu(np.ones((n, n), bool), 1), x, np.float32(-np.inf)).astype(np.float32)
    want, it_want = oracle.closure(op, x)
    got, it = gpu_closure(op, x, cuda)
    assert it == it_want
    np.testing.assert_array_equal(bits(got), bits(want))


def test_directed_cycle_closed_form(cuda):
    n = 300
    x = np.full((n, n), np.inf, np.float32)
    np.fill_diagonal(x, 0)
    for i in range(n):
        x[i, (i + 1) % n] = 1.0
    got, it = gpu_closure("min_plus", x, cuda)
    i, j = np.indices((n, n))
    np.testing.assert_array_equal(got, ((j - i) % n).astype(np.float32))
    assert it == int(np.ceil(np.log2(n - 1))) + 1


def test_convergence_modes(cuda):
    x = datagen.er_graph(200, 0.05, seed=3)
    for conv, mode in (("tol", 1), ("exact", 0)):
        want, it_want = oracle.closure("min_plus", x, tol_mode=mode)
        got, it = gpu_closure("min_plus", x, cuda, conv=conv)
        assert it == it_want
        np.testing.assert_array_equal(bits(got), bits(want))
    # APLP variant on a DAG with max_plus
    n = 150
    y = datagen.closure_graph("max_plus", n, 0.05, seed=5)
    y = np.where(np.triu(np.ones((n, n), bool), 1), y, np.float32(-np.inf)).astype(np.float32)
    want, it_want = oracle.closure("max_plus", y, tol_mode=2)
    got, it = gpu_closure("max_plus", y, cuda, conv="aplp")
    assert it == it_want
    np.testing.assert_array_equal(bits(got), bits(want))


def test_not_converged_reports(cuda):
    n = 64
    x = np.full((n, n), np.inf, np.float32)
    np.fill_diagonal(x, 0)
    for i in range(n - 1):
        x[i, i + 1] = 1.0
    X = torch.from_numpy(x).to(cuda)
    with pytest.raises(s2.NotConverged):
        s2.closure("min_plus", X, max_iter=2)
    X = torch.from_numpy(x).to(cuda)
    assert s2.closure("min_plus", X, max_iter=2, raise_not_converged=False) == 2


def test_or_and_closure(cuda):
    n = 300
    rng = np.random.default_rng(8)
    x = (rng.random((n, n)) < 2.0 / n).astype(np.uint8)
    np.fill_diagonal(x, 1)
    want, it_want = oracle.closure("or_and", x)
    X = torch.from_numpy(x).to(cuda)
    it = s2.closure("or_and", X)
    assert it == it_want
    np.testing.assert_array_equal(X.cpu().numpy(), want)


def _orand_dense_closure(X, max_iter=64):
    """The dense INT8 squaring step repeated to the fixed point (the panel
    step over all rows), as the reference's closure loop runs it."""
    changed = torch.zeros(1, dtype=torch.int32, device=X.device)
    out = torch.empty_like(X)
    it = 0
    while it < max_iter:
        it += 1
        changed.zero_()
        s2.closure_panel_step("or_and", X, X, out, changed)
        X, out = out, X
        if int(changed.item()) == 0:
            break
    return X, it


@pytest.mark.parametrize("case", ["er_deg2", "cycles", "non01", "non01_255", "pitched"])
def test_or_and_closure_sparse_opening(cuda, case):
    """From n = 8192 the or_and closure squares a sparse X as CSR SpGEMM
    steps before the INT8 tensor-core steps: same bits and step count as the
    dense loop ('cycles' converges while still sparse; 'non01' holds bytes
    other than 0 / 1, which the dense step rewrites, so the opening stands
    aside; 'pitched' closes X in place inside a wider, unaligned buffer, where
    the conversion to CSR reads bytes one at a time)."""
    n = 8192
    rng = np.random.default_rng(8192)
    X = torch.zeros((n, n), dtype=torch.uint8, device=cuda)
    if case == "cycles":
        i = torch.arange(n, device=cuda)
        X[i, (i // 8) * 8 + (i + 1) % 8] = 1
    else:
        m = 2 * n
        X[torch.from_numpy(rng.integers(0, n, m)).to(cuda), torch.from_numpy(rng.integers(0, n, m)).to(cuda)] = 1
    X.fill_diagonal_(1)
    if case == "non01":
        X[5, 7] = 2
    if case == "non01_255":
        X[8000, 3] = 255
    want, it_want = _orand_dense_closure(X.clone())
    if case == "pitched":
        buf = torch.zeros((n, n + 5), dtype=torch.uint8, device=cuda)
        buf[:, 1:n + 1] = X
        X = buf[:, 1:n + 1]
    it = s2.closure("or_and", X)
    assert it == it_want
    assert torch.equal(X, want)


def test_or_and_closure_opening_step_cap(cuda):
    """max_iter = 2 inside the or_and closure's sparse opening: NotConverged and
    the dense loop's X after two squarings."""
    n = 8192
    rng = np.random.default_rng(3)
    X = torch.zeros((n, n), dtype=torch.uint8, device=cuda)
    m = 2 * n
    X[torch.from_numpy(rng.integers(0, n, m)).to(cuda), torch.from_numpy(rng.integers(0, n, m)).to(cuda)] = 1
    X.fill_diagonal_(1)
    want, _ = _orand_dense_closure(X.clone(), max_iter=2)
    with pytest.raises(s2.NotConverged):
        s2.closure("or_and", X, max_iter=2)
    assert torch.equal(X, want)
