"""GPU parity: libsimd2 srgemm (through the C ABI) against the CPU oracle.

Min/max semirings and or_and must be bit-exact against host_srgemm semantics.
plus_mul and minus_square run on the tensor cores with BF16 hi/lo operands
(a*b ~= a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32 accumulate).  They are compared
with the FP64 oracle under the forward-error bound

    |D - D64| <= (4 * 2^-16 + 2 * K * 2^-24) * S

where S = sum_k |a_ik||b_kj| + |c_ij| (plus_mul) or 2 sum_k (a_ik^2 + b_kj^2) + |c_ij|
(minus_square): 3 * 2^-16 covers the dropped lo*lo term and the two split
residuals per product, K * 2^-24 the FP32 accumulation.
"""
import os

import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MINMAX = ["min_plus", "max_plus", "max_min", "max_mul", "min_mul", "min_max"]
SUMS = ["plus_mul", "minus_square"]
EPS32 = 2.0 ** -24
SPLIT = 4.0 * 2.0 ** -16  # BF16 hi/lo split error per product (relative to |a||b|)

SHAPES = [(1, 1, 1), (17, 23, 13), (128, 128, 32), (129, 130, 33), (64, 256, 100), (300, 517, 257), (7, 5, 700)]


def bits(x):
    x = np.ascontiguousarray(x)
    return x.view(np.uint32) if x.dtype == np.float32 else x


def run_gpu(op, a, b, c, epi, dev):
    A = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    B = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    C = torch.from_numpy(np.ascontiguousarray(c)).to(dev)
    D = s2.srgemm(op, A, B, C, do_epilogue=epi)
    torch.cuda.synchronize()
    return D.cpu().numpy()


def abs_sum(op, a, b, c, epi):
    a64, b64 = np.abs(a.astype(np.float64)), np.abs(b.astype(np.float64))
    if op == "plus_mul":
        s = a64 @ b64
    else:  # (a-b)^2 <= 2a^2 + 2b^2
        s = 2 * (a64 ** 2).sum(1)[:, None] + 2 * (b64 ** 2).sum(0)[None, :]
    if epi:
        s = s + np.abs(c.astype(np.float64))
    return s


def check_sum_op(op, a, b, c, epi, got):
    want = oracle.srgemm_f64(op, a, b, c, do_epilogue=epi)
    k = a.shape[1]
    bound = (SPLIT + 2.0 * max(k, 1) * EPS32) * abs_sum(op, a, b, c, epi) + 1e-30
    err = np.abs(got.astype(np.float64) - want)
    assert np.all(err <= bound), f"{op}: max err {err.max():.3e}, worst ratio {(err / bound).max():.3f}"


@pytest.mark.parametrize("op", MINMAX + SUMS)
@pytest.mark.parametrize("shape", SHAPES)
def test_srgemm_random_shapes(cuda, op, shape):
    m, n, k = shape
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=m * 131 + n * 7 + k)
    for epi in (False, True):
        got = run_gpu(op, a, b, c, epi, cuda)
        if op in MINMAX:
            want = oracle.srgemm(op, a, b, c, do_epilogue=epi)
            np.testing.assert_array_equal(bits(got), bits(want), err_msg=f"{op} {shape} epi={epi}")
        else:
            check_sum_op(op, a, b, c, epi, got)


@pytest.mark.parametrize("op", oracle.OPS)
def test_srgemm_golden(cuda, op):
    g = np.load(os.path.join(GOLDEN, f"srgemm_{op}.npz"))
    for s in sorted({k.split("_")[0] for k in g.files}):
        a, b, c = g[f"{s}_A"], g[f"{s}_B"], g[f"{s}_C"]
        for epi in (0, 1):
            got = run_gpu(op, a, b, c, bool(epi), cuda)
            if op in SUMS:
                check_sum_op(op, a, b, c, bool(epi), got)
            else:
                np.testing.assert_array_equal(bits(got), bits(g[f"{s}_e{epi}_D"]), err_msg=f"{op} {s} e{epi}")


@pytest.mark.parametrize("dtype", [np.int32, np.uint8])
def test_or_and(cuda, dtype):
    for (m, n, k) in [(1, 1, 1), (33, 65, 17), (200, 130, 300)]:
        a, b, c = datagen.semiring_operands("or_and", m, n, k, seed=k)
        a = (np.random.default_rng(1).random((m, k)) < 0.2).astype(dtype) * 3  # nonzero != 1 is true too
        a, b, c = a.astype(dtype), b.astype(dtype), c.astype(dtype)
        for epi in (False, True):
            got = run_gpu("or_and", a, b, c, epi, cuda)
            want = oracle.srgemm("or_and", a.astype(np.int32), b.astype(np.int32), c.astype(np.int32),
                                 do_epilogue=epi)
            np.testing.assert_array_equal(got.astype(np.int32), want)


@pytest.mark.parametrize("m,n,k,pad,shift", [(70, 300, 200, 20, 0), (33, 130, 100, 5, 1), (129, 64, 17, 0, 0),
                                             (16, 1000, 77, 3, 7)])
def test_or_and_bytes_any_nonzero_strided(cuda, m, n, k, pad, shift):
    """Byte operands whose true entries include bytes with the top bit set
    (0x80, 0xff), B with a pitch past n and a base off the 16-byte boundary
    (B^T is formed 16 bytes at a time where B allows, byte by byte elsewhere),
    ragged k and n: D = A (x) B (+) C against the oracle."""
    rng = np.random.default_rng(m * 7 + n + k)
    vals = np.array([1, 2, 127, 128, 255], np.uint8)
    a = np.where(rng.random((m, k)) < 0.1, rng.choice(vals, (m, k)), 0).astype(np.uint8)
    b = np.where(rng.random((k, n)) < 0.1, rng.choice(vals, (k, n)), 0).astype(np.uint8)
    c = (rng.random((m, n)) < 0.05).astype(np.uint8)
    Bbuf = torch.zeros((k, n + pad + shift), dtype=torch.uint8, device=cuda)
    Bbuf[:, shift:shift + n] = torch.from_numpy(b).to(cuda)
    A, B, C = torch.from_numpy(a).to(cuda), Bbuf[:, shift:shift + n], torch.from_numpy(c).to(cuda)
    for epi in (False, True):
        got = s2.srgemm("or_and", A, B, C, do_epilogue=epi).cpu().numpy()
        want = oracle.srgemm("or_and", a.astype(np.int32), b.astype(np.int32), c.astype(np.int32), do_epilogue=epi)
        np.testing.assert_array_equal(got.astype(np.int32), want)


def test_k_zero_and_empty(cuda):
    for op in MINMAX + SUMS:
        a, b, c = datagen.semiring_operands(op, 9, 11, 0, seed=1)
        got = run_gpu(op, a, b, c, False, cuda)
        want = oracle.srgemm(op, a, b, c, do_epilogue=False)
        np.testing.assert_array_equal(bits(got), bits(want))
        got = run_gpu(op, a, b, c, True, cuda)
        np.testing.assert_array_equal(bits(got), bits(c))
    A = torch.zeros((0, 5), device=cuda)
    B = torch.zeros((5, 3), device=cuda)
    assert s2.srgemm("min_plus", A, B).shape == (0, 3)


def test_strided_and_unaligned_operands(cuda):
    """Row pitches that are not multiples of 4 floats take the packing path."""
    op = "min_plus"
    m, n, k = 70, 90, 45
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=9)
    Abig = torch.full((m, k + 3), 5.0, device=cuda)
    Abig[:, :k] = torch.from_numpy(a).to(cuda)
    Bbig = torch.full((k, n + 1), 5.0, device=cuda)
    Bbig[:, :n] = torch.from_numpy(b).to(cuda)
    Cbig = torch.full((m, n + 5), 5.0, device=cuda)
    Cbig[:, :n] = torch.from_numpy(c).to(cuda)
    Dbig = torch.full((m, n + 7), -1.0, device=cuda)
    s2.srgemm(op, Abig[:, :k], Bbig[:, :n], Cbig[:, :n], do_epilogue=True, D=Dbig[:, :n])
    torch.cuda.synchronize()
    want = oracle.srgemm(op, a, b, c, do_epilogue=True)
    np.testing.assert_array_equal(bits(Dbig[:, :n].cpu().numpy()), bits(want))
    assert torch.all(Dbig[:, n:] == -1.0)  # nothing written past N


def test_in_place_epilogue(cuda):
    """D aliasing C accumulates in place (host_srgemm's D += semantics)."""
    op = "max_plus"
    a, b, c = datagen.semiring_operands(op, 100, 120, 64, seed=4)
    A, B = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
    C = torch.from_numpy(c).to(cuda)
    s2.srgemm(op, A, B, C, do_epilogue=True, D=C)
    torch.cuda.synchronize()
    want = oracle.srgemm(op, a, b, c, do_epilogue=True)
    np.testing.assert_array_equal(bits(C.cpu().numpy()), bits(want))


@pytest.mark.parametrize("op", SUMS + ["or_and"])
def test_full_size_tensor_core_row_sample(cuda, op):
    """4096^3 on the tensor-core paths: FP64-bounded (sums) / exact (or_and) on sampled rows."""
    n = 4096
    a, b, c = datagen.semiring_operands(op, n, n, n, seed=78)
    got = run_gpu(op, a, b, c, True, cuda)
    rows = np.random.default_rng(1).choice(n, size=16, replace=False)
    if op == "or_and":
        want = oracle.srgemm(op, a[rows], b, c[rows], do_epilogue=True)
        np.testing.assert_array_equal(got[rows], want)
    else:
        check_sum_op(op, a[rows], b, c[rows], True, got[rows])
    assert s2.device_status() == 0


def test_minus_square_near_duplicates(cuda):
    """Near-identical points (offset 1e-3) fall in the cancellation band and are recomputed exactly."""
    q, r = datagen.point_cloud(300, 500, 128, seed=3, dup_frac=0.3)
    a, b = q, np.ascontiguousarray(r.T)
    c = np.zeros((300, 500), np.float32)
    got = run_gpu("minus_square", a, b, c, False, cuda)
    want = oracle.srgemm_f64("minus_square", a, b)
    small = want < 1e-2
    assert small.sum() > 50
    rel = np.abs(got[small] - want[small]) / want[small]
    assert rel.max() < 1e-4, rel.max()
    check_sum_op("minus_square", a, b, c, False, got)


@pytest.mark.parametrize("op", MINMAX)
def test_full_size_row_sample(cuda, op):
    """4096^3 (the nine-semiring sweep size): bit-exact on a sample of rows."""
    n = 4096
    a, b, c = datagen.semiring_operands(op, n, n, n, seed=77)
    got = run_gpu(op, a, b, c, True, cuda)
    rows = np.random.default_rng(0).choice(n, size=24, replace=False)
    want = oracle.srgemm(op, a[rows], b, c[rows], do_epilogue=True)
    np.testing.assert_array_equal(bits(got[rows]), bits(want))
    assert s2.device_status() == 0


def test_min_plus_8192_row_sample(cuda):
    """min_plus at 8192^3 (the size of the reference's srgemm micro-benchmark,
    micro_bench/srgemm_bench.cu:252) on the sweep's value distribution:
    bit-exact against host_srgemm on 32 sampled rows -- the reference's own
    compiled header where it was built, else the restatement pinned to it."""
    n = 8192
    a, b, c = datagen.semiring_operands("min_plus", n, n, n, seed=8192)
    got = run_gpu("min_plus", a, b, c, True, cuda)
    rows = np.random.default_rng(8192).choice(n, size=32, replace=False)
    use_ref = oracle.ref_lib() is not None
    want = oracle.srgemm("min_plus", a[rows], b, c[rows], do_epilogue=True, use_ref=use_ref)
    np.testing.assert_array_equal(bits(got[rows]), bits(want))
    assert np.isfinite(got[rows]).mean() > 0.99  # 20 % identities in A and B still leave finite minima
    assert s2.device_status() == 0


@pytest.mark.parametrize("op", ["max_min", "min_max"])
def test_selection_fp16_and_fp32_paths(cuda, op):
    """max_min / min_max take the packed-FP16 kernel when every A and B entry
    is an FP16 value, else the FP32 kernel; both must give host_srgemm's bits."""
    rng = np.random.default_rng(12)
    m, n, k = 257, 190, 333
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=12)  # integer-valued: FP16 path
    cases = [("fp16-exact", a, b)]
    af = rng.random((m, k), dtype=np.float32)  # generic floats: FP32 path
    bf = rng.random((k, n), dtype=np.float32)
    cases.append(("generic", af, bf))
    a1 = a.copy()
    a1[5, 7] = np.float32(1.0001)  # one non-FP16 entry switches the whole call to FP32
    cases.append(("one-off", a1, b))
    b2 = b.copy()
    b2[3, 4] = np.float32(70000.0)  # above the FP16 range
    cases.append(("overflow", a, b2))
    for name, x, y in cases:
        for epi in (False, True):
            got = run_gpu(op, x, y, c, epi, cuda)
            want = oracle.srgemm(op, x, y, c, do_epilogue=epi)
            np.testing.assert_array_equal(bits(got), bits(want), err_msg=f"{op} {name} epi={epi}")


@pytest.mark.parametrize("op", ["plus_mul", "minus_square", "or_and"])
@pytest.mark.parametrize("shape", [(1024, 1024, 2048), (4096, 4096, 256), (130, 300, 700), (4096, 1200, 512),
                                   (2560, 2560, 384)])
def test_tensor_core_partial_rounds(cuda, op, shape):
    """Shapes that leave the persistent tensor-core grid partly idle (fewer
    tiles than SMs; the last round of 4096 x 4096, 4096 x 1200 and 2560 x 2560
    on the SM-pair kernel, run as 256 x 128 half tiles, one of them past a
    ragged column edge; ragged edges): the oracle's result (or_and exactly) on
    rows sampled across the output."""
    M, N, K = shape
    a, b, c = datagen.semiring_operands(op, M, N, K, seed=M + K)
    A, B, C = (torch.from_numpy(x).to(cuda) for x in (a, b, c))
    got = s2.srgemm(op, A, B, C, do_epilogue=True).cpu().numpy()
    rows = np.unique(np.linspace(0, M - 1, 40).astype(int))
    if op == "or_and":
        want = oracle.srgemm(op, a[rows], b, c[rows], do_epilogue=True)
        assert np.array_equal(got[rows], want)
        return
    want = oracle.srgemm_f64(op, a[rows], b, c[rows], do_epilogue=True)
    g = got[rows].astype(np.float64)
    if op == "plus_mul":
        S = np.abs(a[rows]).astype(np.float64) @ np.abs(b).astype(np.float64) + np.abs(c[rows])
    else:
        S = ((a[rows].astype(np.float64) ** 2).sum(1)[:, None] + (b.astype(np.float64) ** 2).sum(0)[None, :]) * 2 \
            + np.abs(c[rows])
    assert np.all(np.abs(g - want) <= (4 * 2.0 ** -16 + 2 * K * 2.0 ** -24) * S + 1e-6)
    assert s2.device_status() == 0


@pytest.mark.parametrize("op", SUMS)
def test_summing_semirings_error_level(cuda, op):
    """The BF16 hi/lo path's measured error against FP64, at the sweep's
    values and K = 4096, stays at the level the split gives, far inside the
    worst-case bound above: per product the dropped lo*lo term and the two
    split residuals are each at most 2^-18 |a||b|, and FP32 accumulation over
    K terms of random sign adds about sqrt(K) * 2^-24 (4x margin here).  A
    split that lost its hi*lo or lo*hi term would miss this by orders of
    magnitude."""
    m, n, k = 384, 512, 4096
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=4096 + len(op))
    got = run_gpu(op, a, b, c, True, cuda).astype(np.float64)
    want = oracle.srgemm_f64(op, a, b, c, do_epilogue=True)
    S = abs_sum(op, a, b, c, True)
    level = 3 * 2.0 ** -18 + 4 * np.sqrt(k) * 2.0 ** -24
    ratio = (np.abs(got - want) / S).max()
    assert ratio <= level, (op, ratio, level)
