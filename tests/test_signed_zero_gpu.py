"""Signed zeros in max_mul / min_mul (kernel/host_srgemm.h:53-70).

host_srgemm folds products with std::max(D, p) = (D < p ? p : D) (std::min
alike), so among products that tie at zero the first one in k order keeps
its sign.  A -0.0 product arises only as a zero times a negative operand.
The device folds products in another grouping, so the library's exactness
precondition for these two semirings is: no product is -0.0 (no zero operand
alongside negative ones).  These tests pin what holds on either side of it:

* operands in [0, 1] that include exact zeros (the reference apps' maxrp /
  minrp regime): bit-exact through srgemm, the closure and the batched
  closure, with the same step counts;
* operands in [-1, 1] that include exact zeros: the same values everywhere
  (a bit can differ only in the sign of a zero result), and the closures
  under the reference's |delta| > 1e-4 change test take the same steps.
"""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2

pytestmark = pytest.mark.gpu
OPS = ["max_mul", "min_mul"]


def _signed(rng, shape, zero_frac, lo=-1.0):
    x = (lo + (1.0 - lo) * rng.random(shape, dtype=np.float32)).astype(np.float32)
    x[rng.random(shape) < zero_frac] = 0.0
    x[x == 0] = 0.0  # +0 only: the precondition excludes -0.0 operands
    return x


def _same_values(got, want, what):
    assert np.array_equal(got, want), f"{what}: values differ"  # +0 == -0 here
    diff = got.view(np.uint32) != want.view(np.uint32)
    assert np.all(want[diff] == 0), f"{what}: a nonzero result differs in its bits"
    return int(diff.sum())


@pytest.mark.parametrize("op", OPS)
def test_srgemm_nonnegative_with_zeros_is_bit_exact(cuda, op):
    rng = np.random.default_rng(5)
    for (m, n, k) in [(129, 130, 257), (64, 300, 8), (1000, 257, 64)]:
        a, b, c = (_signed(rng, s, 0.3, lo=0.0) for s in ((m, k), (k, n), (m, n)))
        for epi in (False, True):
            A, B, C = (torch.from_numpy(x).to(cuda) for x in (a, b, c))
            got = s2.srgemm(op, A, B, C, do_epilogue=epi).cpu().numpy()
            want = oracle.srgemm(op, a, b, c, do_epilogue=epi)
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=f"{op} {m}x{n}x{k}")


@pytest.mark.parametrize("op", OPS)
def test_srgemm_signed_with_zeros_same_values(cuda, op):
    """Products of both zero signs tie at a zero result: short K, and one
    operand's signs chosen so that the extreme product is often zero."""
    rng = np.random.default_rng(6)
    zero_results = 0
    for (m, n, k) in [(200, 180, 4), (128, 256, 16), (333, 129, 300)]:
        a = _signed(rng, (m, k), 0.4, lo=0.0)
        b = _signed(rng, (k, n), 0.1)
        if op == "max_mul":  # nonpositive products except where b > 0
            b = np.where(rng.random(b.shape) < 0.8, -np.abs(b), b).astype(np.float32)
        else:
            b = np.where(rng.random(b.shape) < 0.8, np.abs(b), b).astype(np.float32)
        c = _signed(rng, (m, n), 0.2)
        for epi in (False, True):
            A, B, C = (torch.from_numpy(x).to(cuda) for x in (a, b, c))
            got = s2.srgemm(op, A, B, C, do_epilogue=epi).cpu().numpy()
            want = oracle.srgemm(op, a, b, c, do_epilogue=epi)
            _same_values(got, want, f"{op} {m}x{n}x{k} epi={epi}")
            zero_results += int((want == 0).sum())
    assert zero_results > 1000  # the zero ties were exercised


def _graph(rng, n, lo):
    x = _signed(rng, (n, n), 0.3, lo=lo)
    x[rng.random((n, n)) < 0.5] = 0.0
    np.fill_diagonal(x, 1.0)
    return x.astype(np.float32)


@pytest.mark.parametrize("op", OPS)
def test_closures_nonnegative_with_zeros_bit_exact(cuda, op):
    rng = np.random.default_rng(7)
    graphs = [_graph(rng, n, 0.0) for n in (40, 130, 300)]
    for x in graphs:
        X = torch.from_numpy(x).to(cuda)
        it = s2.closure(op, X)
        want, it_want = oracle.closure(op, x)
        assert it == it_want
        np.testing.assert_array_equal(X.cpu().numpy().view(np.uint32), want.view(np.uint32))
    mats = [torch.from_numpy(x).to(cuda) for x in graphs]
    its = s2.closure_batched(op, mats)
    for x, m, it in zip(graphs, mats, its):
        want, it_want = oracle.closure(op, x)
        assert it == it_want
        np.testing.assert_array_equal(m.cpu().numpy().view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("op", OPS)
def test_closures_signed_with_zeros_same_values(cuda, op):
    rng = np.random.default_rng(8)
    graphs = [_graph(rng, n, -1.0) for n in (40, 130, 300)]
    for x in graphs:
        X = torch.from_numpy(x).to(cuda)
        it = s2.closure(op, X, conv="tol")
        want, it_want = oracle.closure(op, x, tol_mode=1)
        assert it == it_want
        _same_values(X.cpu().numpy(), want, f"{op} closure n={x.shape[0]}")
    mats = [torch.from_numpy(x).to(cuda) for x in graphs]
    its = s2.closure_batched(op, mats, conv="tol")
    for x, m, it in zip(graphs, mats, its):
        want, it_want = oracle.closure(op, x, tol_mode=1)
        assert it == it_want
        _same_values(m.cpu().numpy(), want, f"{op} batched n={x.shape[0]}")
