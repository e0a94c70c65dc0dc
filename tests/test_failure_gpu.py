"""Failure detection without a GPU fault.

Every wait in the kernels is bounded; when a wait runs out the kernel records
SIMD2_ERR_TIMEOUT and a wait-site id instead of hanging.  The self-test kernel
waits on a barrier nothing completes (short limit) and the host reads the
status; the device must stay usable afterwards.  Host-side failures (bad
arguments, non-convergence) are checked too.
"""
import ctypes

import pytest
import torch

import simd2_b200 as s2

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_device_survives(cuda):
    L = s2.lib()
    assert s2.device_status() == 0
    assert L.simd2_selftest_timeout(20000) == 0  # 20 ms wait that runs out
    assert s2.device_status() == 5  # SIMD2_ERR_TIMEOUT, read and cleared
    assert L.simd2_timeout_site() == 99
    assert s2.device_status() == 0
    # the context is still usable
    A = torch.rand((64, 64), device=cuda)
    D = s2.srgemm("min_plus", A, A)
    torch.cuda.synchronize()
    assert torch.isfinite(D).all()


def test_host_side_errors(cuda):
    L = s2.lib()
    assert L.simd2_selftest_timeout(0) == 1
    A = torch.zeros((4, 4), device=cuda)
    with pytest.raises(TypeError):
        s2.srgemm("or_and", A, A)  # float tensors for or_and: rejected, nothing launched
    # invalid leading dimension straight through the C ABI
    P = ctypes.c_void_p
    assert L.simd2_srgemm(0, 4, 4, 4, P(A.data_ptr()), 2, P(A.data_ptr()), 4, None, 4, P(A.data_ptr()), 4, 0,
                          None) == 1
    with pytest.raises(ValueError):
        s2.srgemm("min_plus", A, torch.zeros((5, 4), device=cuda))
    assert s2.device_status() == 0
