"""Generate the golden srgemm / closure fixtures from the reference itself.

Runs escalab/SIMD2's own ``mmo::host_srgemm`` (kernel/host_srgemm.h), compiled
unchanged into oracle/_ref/libref.so by oracle/Makefile, on small seeded
inputs and stores inputs + outputs as .npz files next to this script.  The
fixtures pin the C restatement (oracle/simd2_oracle.c) and the GPU kernels
on machines where the reference tree is absent.

    python tests/golden/make_golden.py      (needs oracle/_ref/libref.so)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from simd2_b200 import datagen  # noqa: E402

SHAPES = [(17, 23, 13), (32, 40, 33), (5, 1, 64), (64, 3, 7)]


def main():
    if oracle.ref_lib() is None:
        raise SystemExit("oracle/_ref/libref.so missing: build it with `make -C oracle` where the reference exists")
    for op in oracle.OPS:
        out = {}
        for si, (m, n, k) in enumerate(SHAPES):
            a, b, c = datagen.semiring_operands(op, m, n, k, seed=1000 + si, identity_frac=0.2)
            if op == "or_and":
                a, b, c = a.astype(np.int32), b.astype(np.int32), c.astype(np.int32)
            for epi in (0, 1):
                d = oracle.srgemm(op, a, b, c, do_epilogue=bool(epi), use_ref=True, threads=1)
                out[f"s{si}_e{epi}_D"] = d
            out[f"s{si}_A"], out[f"s{si}_B"], out[f"s{si}_C"] = a, b, c
        np.savez_compressed(os.path.join(HERE, f"srgemm_{op}.npz"), **out)
    # closure: APSP on a 48-node directed ER graph, iterated with the reference
    # host_srgemm exactly as apps/apsp/cuASR/apsp_cuASR.cu:42-54 does.
    for op in ("min_plus", "max_min"):
        x0 = datagen.closure_graph(op, 48, 0.08, seed=7)
        x = x0.copy()
        it = 0
        while it < 500:
            it += 1
            xn = oracle.srgemm(op, x, x, x, do_epilogue=True, use_ref=True, threads=1)
            same = np.array_equal(xn.view(np.uint32), x.view(np.uint32))
            x = xn
            if same:
                break
        np.savez_compressed(os.path.join(HERE, f"closure_{op}.npz"), X0=x0, X=x, iters=np.int32(it))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
