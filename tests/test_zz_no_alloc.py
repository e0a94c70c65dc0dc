"""simd2_srgemm_noalloc: the srgemm entry point that allocates nothing.

It exists for callers that must not call cudaMalloc (a caller-owned pool or
allocator that forbids side allocations, latency-critical loops, processes
that already placed all device memory).  Its scratch is one fixed device
array shared by every call, so these tests make two calls in a row -- the
second on a different semiring and a smaller problem, so that bytes left by
the first call sit in the scratch -- and compare each result with the
allocating entry point simd2_srgemm and with the CPU oracle, bit for bit
(the min/max semirings are exact).  One more test checks the property the
entry point exists for: a call on a stream the library has never seen (so
no workspace of its own) leaves the device's free memory unchanged.  The
file sorts last so that a first-failure run has already run every other
test.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20
ERR_UNSUPPORTED = 2
ERR_SCRATCH_LIMIT = 8


def _lib():
    L = s2.lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    L.simd2_srgemm_noalloc.argtypes = [I, I, I, I, P, I, P, I, P, I, P, I, I, P]
    L.simd2_srgemm_noalloc.restype = I
    return L


def _call(fn, op, A, B, C, D, epi):
    M, K = A.shape
    N = B.shape[1]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return fn(s2.OP_ID[op], M, N, K, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), C.data_ptr(),
              C.stride(0), D.data_ptr(), D.stride(0), int(epi), stream)


def _case(L, op, m, n, k, seed, epi, dev, a_pitch=None):
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=seed)
    if a_pitch is None:
        A = torch.from_numpy(a).to(dev)
    else:  # rows of A not 16-byte aligned: the scratch also holds a packed copy of A
        Abig = torch.zeros((m, a_pitch), dtype=torch.float32, device=dev)
        Abig[:, :k] = torch.from_numpy(a).to(dev)
        A = Abig[:, :k]
    B = torch.from_numpy(b).to(dev)
    C = torch.from_numpy(c).to(dev)
    D_ref = torch.full((m, n), 7.0, device=dev)
    D_new = torch.full((m, n), -7.0, device=dev)
    assert _call(L.simd2_srgemm, op, A, B, C, D_ref, epi) == 0
    assert _call(L.simd2_srgemm_noalloc, op, A, B, C, D_new, epi) == 0
    torch.cuda.synchronize()
    got = D_new.cpu().numpy()
    np.testing.assert_array_equal(got.view(np.uint32), D_ref.cpu().numpy().view(np.uint32),
                                  err_msg=f"{op} {m}x{n}x{k}")
    want = oracle.srgemm(op, a, b, c, do_epilogue=epi)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=f"{op} {m}x{n}x{k} vs oracle")


def test_noalloc_matches_allocating_entry_two_calls_in_a_row(cuda):
    L = _lib()
    # call 1: fills most of the scratch (roundup(K,32) * roundup(N,128) * 4 = 2304 * 1536 * 4 = 13.5 MiB)
    _case(L, "min_plus", 1000, 1500, 2300, seed=21, epi=True, dev=cuda)
    # call 2: another semiring on a smaller problem reads over the first call's leftovers
    _case(L, "max_min", 300, 200, 999, seed=22, epi=False, dev=cuda)
    assert s2.device_status() == 0


def test_noalloc_packed_a_and_other_semirings(cuda):
    L = _lib()
    _case(L, "max_plus", 257, 129, 131, seed=23, epi=True, dev=cuda, a_pitch=133)
    _case(L, "min_mul", 64, 64, 64, seed=24, epi=True, dev=cuda)


def test_noalloc_allocates_nothing(cuda):
    """A call on a fresh stream (one the library holds no workspace for) must
    not change the device's free memory: the allocating entry point would
    create a workspace for that stream here.  The first call, on the default
    stream, loads the kernels and places the scratch array."""
    L = _lib()
    op, m, n, k = "min_plus", 300, 400, 500
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=25)
    A, B, C = (torch.from_numpy(x).to(cuda) for x in (a, b, c))
    D = torch.empty((m, n), device=cuda)
    assert _call(L.simd2_srgemm_noalloc, op, A, B, C, D, True) == 0
    torch.cuda.synchronize()
    fresh = torch.cuda.Stream()
    free_before = torch.cuda.mem_get_info()[0]
    with torch.cuda.stream(fresh):
        for _ in range(2):
            assert _call(L.simd2_srgemm_noalloc, op, A, B, C, D, True) == 0
    fresh.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before, (free_before, free_after)
    want = oracle.srgemm(op, a, b, c, do_epilogue=True)
    np.testing.assert_array_equal(D.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_noalloc_rejects_oversize_and_unsupported(cuda):
    L = _lib()
    n = 4096  # 4096 x 4096 x 4 bytes of B' = 64 MiB > 16 MiB
    A = torch.zeros((8, n), device=cuda)
    B = torch.zeros((n, n), device=cuda)
    C = torch.zeros((8, n), device=cuda)
    D = torch.zeros((8, n), device=cuda)
    assert _call(L.simd2_srgemm_noalloc, "min_plus", A, B, C, D, True) == ERR_SCRATCH_LIMIT
    A = torch.zeros((4, 4), device=cuda)
    assert _call(L.simd2_srgemm_noalloc, "plus_mul", A, A, A, A.clone(), False) == ERR_UNSUPPORTED
