"""A reference-style closure app compiled against simd2_cuasr.h runs on libsimd2."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from simd2_b200 import build, datagen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cuasr_style_app(cuda, tmp_path):
    lib = build.build()
    exe = tmp_path / "cuasr_app"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "compat", "cuasr_app.cu"), "-o", str(exe), "-L", os.path.dirname(lib),
           "-lsimd2", f"-Xlinker=-rpath,{os.path.dirname(lib)}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    v = 200
    x = datagen.er_graph(v, 0.03, seed=5)
    x[~np.isfinite(x)] = np.float32(3.4028234663852886e38)  # the apps' FLT_MAX fill
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([v], np.int32).tofile(f)
        x.tofile(f)
    res = subprocess.run([str(exe), str(inp), str(outp)], capture_output=True, text=True)
    assert res.returncode == 0, (res.returncode, res.stdout, res.stderr)
    data = np.fromfile(outp, dtype=np.float32)
    iters = data[:1].view(np.int32)[0]
    dist = data[1:1 + v * v].reshape(v, v)
    r1 = data[1 + v * v:1 + v * v + 256].reshape(16, 16)
    r2 = data[1 + v * v + 256:].reshape(16, 16)
    want, it_want = oracle.closure("min_plus", x, tol_mode=1)
    assert iters == it_want
    np.testing.assert_array_equal(dist.view(np.uint32), want.view(np.uint32))
    a = x[:16, :16].copy()
    a[a > 1e30] = 60000.0
    np.testing.assert_array_equal(r1, oracle.srgemm("min_plus", a, a))
    ah = a.astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(r2, oracle.srgemm("min_plus", ah, ah))


def test_pld_knn_mxu(cuda, tmp_path):
    """The PLD caller's knn_mxu through simd2_cuasr.h: the reference's point
    distribution (10 * uniform, apps/pld/cuASR/test.cpp:13-32) and layouts;
    indices [k][query_nb] against the oracle (the reference's own test asks
    90 % of them right, apps/pld/cuASR/test.cpp:95-115), distances within the
    k-NN error bound."""
    lib = build.build()
    exe = tmp_path / "pld_app"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "compat", "pld_app.cu"), "-o", str(exe), "-L", os.path.dirname(lib),
           "-lsimd2", f"-Xlinker=-rpath,{os.path.dirname(lib)}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    rng = np.random.default_rng(1024)
    ref_nb, query_nb, dim, k = 4096, 777, 64, 16
    ref = (10.0 * rng.random((dim, ref_nb))).astype(np.float32)    # [dim][ref_nb]
    query = (10.0 * rng.random((dim, query_nb))).astype(np.float32)  # [dim][query_nb]
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([ref_nb, query_nb, dim, k], np.int32).tofile(f)
        ref.tofile(f)
        query.tofile(f)
    res = subprocess.run([str(exe), str(inp), str(outp)], capture_output=True, text=True)
    assert res.returncode == 0, (res.returncode, res.stdout, res.stderr)
    data = np.fromfile(outp, dtype=np.uint8)
    dist = data[: query_nb * k * 4].view(np.float32).reshape(k, query_nb)
    index = data[query_nb * k * 4:].view(np.int32).reshape(k, query_nb)
    want_d, want_i, want_sq = oracle.knn(np.ascontiguousarray(query.T), np.ascontiguousarray(ref.T), k)
    assert (index.T == want_i).mean() >= 0.99
    nq = (query.T.astype(np.float64) ** 2).sum(1)[:, None]
    bound = (4 * 2.0 ** -16 + 2 * dim * 2.0 ** -24) * 2 * (nq + (ref.T.astype(np.float64) ** 2).sum(1).max())
    assert np.all(np.abs(dist.T.astype(np.float64) ** 2 - want_sq) <= bound + 1e-6 * want_sq)
