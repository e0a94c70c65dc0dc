"""The CPU oracle pinned against the reference's own host_srgemm.

Golden fixtures (tests/golden/*.npz) were produced by escalab/SIMD2's
mmo::host_srgemm (kernel/host_srgemm.h:17-49) compiled unchanged; see
tests/golden/make_golden.py.  The restatement must match them bit for bit
for all nine semirings (it keeps the k order, so even the summing ones match).
"""
import os

import numpy as np
import pytest

import oracle
from simd2_b200 import datagen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def bits(x):
    x = np.ascontiguousarray(x)
    return x.view(np.uint32) if x.dtype == np.float32 else x


@pytest.mark.parametrize("op", oracle.OPS)
def test_restatement_matches_golden(op):
    g = np.load(os.path.join(GOLDEN, f"srgemm_{op}.npz"))
    shapes = sorted({k.split("_")[0] for k in g.files})
    assert shapes
    for s in shapes:
        a, b, c = g[f"{s}_A"], g[f"{s}_B"], g[f"{s}_C"]
        for epi in (0, 1):
            d = oracle.srgemm(op, a, b, c, do_epilogue=bool(epi), threads=3)
            np.testing.assert_array_equal(bits(d), bits(g[f"{s}_e{epi}_D"]), err_msg=f"{op} {s} epi={epi}")


@pytest.mark.parametrize("op", ["min_plus", "max_min"])
def test_closure_matches_golden(op):
    g = np.load(os.path.join(GOLDEN, f"closure_{op}.npz"))
    x, it = oracle.closure(op, g["X0"])
    assert it == int(g["iters"])
    np.testing.assert_array_equal(bits(x), bits(g["X"]))


@pytest.mark.skipif(oracle.ref_lib() is None, reason="reference host_srgemm not built here")
@pytest.mark.parametrize("op", oracle.OPS)
def test_restatement_matches_reference_live(op):
    rng = np.random.default_rng(5)
    for trial in range(3):
        m, n, k = (int(v) for v in rng.integers(1, 70, size=3))
        a, b, c = datagen.semiring_operands(op, m, n, k, seed=trial)
        if op == "or_and":
            a, b, c = a.astype(np.int32), b.astype(np.int32), c.astype(np.int32)
        for epi in (False, True):
            want = oracle.srgemm(op, a, b, c, do_epilogue=epi, use_ref=True, threads=2)
            got = oracle.srgemm(op, a, b, c, do_epilogue=epi, threads=4)
            np.testing.assert_array_equal(bits(got), bits(want))


def test_u8_or_and_equals_i32():
    a, b, c = datagen.semiring_operands("or_and", 40, 50, 60, seed=3)
    a[a > 0] = 7  # any nonzero byte is true
    d8 = oracle.srgemm("or_and", a, b, c, do_epilogue=True)
    d32 = oracle.srgemm("or_and", a.astype(np.int32), b.astype(np.int32), c.astype(np.int32), do_epilogue=True)
    np.testing.assert_array_equal(d8.astype(np.int32), d32)


# --- closed-form graphs (the idea of the FW baselines' known-answer tests) ---

def test_closure_directed_cycle():
    n = 37
    x = np.full((n, n), np.inf, np.float32)
    np.fill_diagonal(x, 0)
    for i in range(n):
        x[i, (i + 1) % n] = 1.0
    d, it = oracle.closure("min_plus", x)
    i, j = np.indices((n, n))
    np.testing.assert_array_equal(d, ((j - i) % n).astype(np.float32))
    # ceil(log2(n-1)) squarings reach every distance, plus one unchanged step
    assert it == int(np.ceil(np.log2(n - 1))) + 1


def test_closure_complete_graph_and_empty_graph():
    n = 16
    kn = np.ones((n, n), np.float32)
    np.fill_diagonal(kn, 0)
    d, it = oracle.closure("min_plus", kn)
    np.testing.assert_array_equal(d, kn)
    assert it == 1
    empty = np.full((n, n), np.inf, np.float32)
    np.fill_diagonal(empty, 0)
    d, it = oracle.closure("min_plus", empty)
    np.testing.assert_array_equal(d, empty)
    assert it == 1


def test_closure_k1_pairs():
    # disjoint edges (2i, 2i+1) of weight 3: distances stay within each pair
    n = 20
    x = np.full((n, n), np.inf, np.float32)
    np.fill_diagonal(x, 0)
    for i in range(0, n, 2):
        x[i, i + 1] = x[i + 1, i] = 3.0
    d, _ = oracle.closure("min_plus", x)
    np.testing.assert_array_equal(d, x)


def test_closure_tolerance_modes():
    x = datagen.er_graph(40, 0.1, seed=2)
    d0, it0 = oracle.closure("min_plus", x, tol_mode=0)
    d1, it1 = oracle.closure("min_plus", x, tol_mode=1)
    np.testing.assert_array_equal(d0, d1)  # integer weights: both tests agree
    assert it0 == it1


def test_knn_oracle_brute_force():
    q, r = datagen.point_cloud(23, 101, 9, seed=4, dup_frac=0.2)
    dist, idx, sq = oracle.knn(q, r, 5)
    full = ((q[:, None, :].astype(np.float64) - r[None, :, :]) ** 2).sum(-1)
    order = np.lexsort((np.broadcast_to(np.arange(101), full.shape), full), axis=1)[:, :5]
    np.testing.assert_array_equal(idx, order)
    np.testing.assert_allclose(sq, np.take_along_axis(full, order, 1), rtol=1e-12)
    np.testing.assert_allclose(dist, np.sqrt(np.take_along_axis(full, order, 1)), rtol=1e-6)
