"""GPU parity of the FP16-input entry (simd2_srgemm_f16, the library behind the
reference's ``tensor_srgemm``, kernel/tensor_srgemm.cuh:197-218) for all nine
opcodes on shapes that are multiples of 16, against the CPU oracle run on the
widened FP16 values: bit-exact for the six min/max semirings and or_and (any
nonzero half is true), within the FP64 error bound of the tensor-core path for
plus_mul and minus_square."""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu
MINMAX = ["min_plus", "max_plus", "max_min", "max_mul", "min_mul", "min_max"]
SHAPES = [(16, 16, 16), (64, 48, 32), (128, 256, 96), (272, 160, 528)]


def _inputs(op, m, n, k, seed):
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=seed)
    if op == "or_and":
        rng = np.random.default_rng(seed)
        a = a.astype(np.float32) * rng.choice(np.array([1.0, 3.0, -2.0, 0.5], np.float32), size=a.shape)
        b = (rng.random(b.shape) < 0.3).astype(np.float32)
        c = c.astype(np.float32)
    ah = a.astype(np.float16)
    bh = b.astype(np.float16)
    return ah, bh, c.astype(np.float32)


@pytest.mark.parametrize("op", s2.OPS)
@pytest.mark.parametrize("shape", SHAPES)
def test_f16_entry_all_opcodes(cuda, op, shape):
    m, n, k = shape
    ah, bh, c = _inputs(op, m, n, k, seed=m + 3 * n + 7 * k + s2.OP_ID[op])
    a, b = ah.astype(np.float32), bh.astype(np.float32)  # exact widening
    A, B = torch.from_numpy(ah).to(cuda), torch.from_numpy(bh).to(cuda)
    C = torch.from_numpy(c).to(cuda)
    for epi in (False, True):
        got = s2.srgemm_f16(op, A, B, C, do_epilogue=epi).cpu().numpy()
        if op in MINMAX:
            want = oracle.srgemm(op, a, b, c, do_epilogue=epi)
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=f"{op} {shape} {epi}")
        elif op == "or_and":
            want = oracle.srgemm("or_and", (a != 0).astype(np.int32), (b != 0).astype(np.int32),
                                 (c != 0).astype(np.int32), do_epilogue=epi)
            np.testing.assert_array_equal(got, want.astype(np.float32), err_msg=f"{shape} {epi}")
        else:
            want = oracle.srgemm_f64(op, a, b, c, do_epilogue=epi)
            a64, b64 = np.abs(a.astype(np.float64)), np.abs(b.astype(np.float64))
            if op == "plus_mul":
                S = a64 @ b64
            else:
                S = 2 * (a64 ** 2).sum(1)[:, None] + 2 * (b64 ** 2).sum(0)[None, :]
            if epi:
                S = S + np.abs(c.astype(np.float64))
            err = np.abs(got.astype(np.float64) - want)
            assert np.all(err <= (4 * 2.0 ** -16 + 2 * k * 2.0 ** -24) * S + 1e-30), (op, shape, epi, err.max())
    assert s2.device_status() == 0
