"""The drop-in closure app driver against the oracle, with the reference apps'
input formats, fill conventions, change tests and output line."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle
from simd2_b200 import build

pytestmark = pytest.mark.gpu
FLT_MAX = np.float32(3.4028234663852886e38)


@pytest.fixture(scope="module")
def app():
    return build.build_app()


def run(app, args, stdin=None, tmp=None):
    out = os.path.join(tmp, "res.bin")
    res = subprocess.run([app, *args, "--repeat", "2", "--out", out], input=stdin, capture_output=True, text=True)
    assert res.returncode == 0, (res.returncode, res.stderr)
    ms, it = res.stdout.split()
    assert float(ms) >= 0
    data = np.fromfile(out, dtype=np.float32)
    v = data[:1].view(np.int32)[0]
    return int(it), data[1:].reshape(v, v)


def edge_text(v, edges):
    return f"{v} {len(edges)}\n" + "".join(f"{a} {b} {w}\n" for a, b, w in edges)


def oracle_closure(op, x, mode):
    return oracle.closure(op, x, tol_mode=mode)


CASES = {
    # app: (op, fill, diag or None, tol_mode, weight sampler, dag)
    "apsp": ("min_plus", FLT_MAX, 0.0, 1, lambda r: float(r.integers(1, 101)), False),
    "aplp": ("max_plus", -FLT_MAX, None, 2, lambda r: float(r.integers(1, 101)), True),
    "mcp": ("max_min", -FLT_MAX, -FLT_MAX, 1, lambda r: float(r.integers(1, 101)), False),
    "maxrp": ("max_mul", np.float32(0.0), None, 1, lambda r: round(float(r.uniform(0.05, 1.0)), 4), False),
    "minrp": ("min_mul", FLT_MAX, None, 1, lambda r: round(float(r.uniform(1.0, 3.0)), 4), False),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_edge_list_apps(cuda, app, tmp_path, name):
    op, fill, diag, mode, sample, dag = CASES[name]
    rng = np.random.default_rng(len(name))
    v = 150
    edges = []
    for _ in range(600):
        a, b = int(rng.integers(v)), int(rng.integers(v))
        if a == b or (dag and a > b):
            continue
        edges.append((a, b, sample(rng)))
    x = np.full((v, v), fill, np.float32)
    for a, b, w in edges:
        x[a, b] = np.float32(int(w)) if name == "aplp" else np.float32(w)
    if diag is not None:
        np.fill_diagonal(x, np.float32(diag))
    it, got = run(app, [name, "-f"], stdin=edge_text(v, edges), tmp=str(tmp_path))
    want, it_want = oracle_closure(op, x, mode)
    assert it == it_want
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def libc_rgg(v, density, w, directed):
    """The generated-graph mode's draws, through the C library's own rand()."""
    libc = ctypes.CDLL("libc.so.6")
    libc.rand.restype = ctypes.c_int
    libc.srand(7)
    RAND_MAX = 2147483647
    g = np.zeros((v, v), np.float32)
    for i in range(v):
        for j in range(v):
            if i == j:
                continue
            if directed or j > i:
                weight = np.float32(np.float32(libc.rand()) / np.float32(RAND_MAX / w))
                has = np.float32(np.float32(libc.rand()) / np.float32(RAND_MAX / 1))
                val = weight if has < np.float32(density) else FLT_MAX
                g[i, j] = val
                if not directed:
                    g[j, i] = val
    return g


def test_generated_apsp(cuda, app, tmp_path):
    v = 160
    x = libc_rgg(v, 0.05, 100.0, directed=False)
    it, got = run(app, ["apsp", str(v), "0.05", "100"], tmp=str(tmp_path))
    want, it_want = oracle_closure("min_plus", x, 1)
    assert it == it_want
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_generated_gtc(cuda, app, tmp_path):
    v = 200
    g = libc_rgg(v, 0.01, 10.0, directed=True)
    t = (g < FLT_MAX - 100).astype(np.uint8)
    np.fill_diagonal(t, 1)
    it, got = run(app, ["gtc", str(v), "0.01"], tmp=str(tmp_path))
    want, it_want = oracle.closure("or_and", t)
    assert it == it_want
    np.testing.assert_array_equal(got.astype(np.uint8), want)


def test_mst_pbbs_file(cuda, app, tmp_path):
    rng = np.random.default_rng(4)
    v = 120
    lines = ["WeightedEdgeArray"]
    x = np.zeros((v, v), np.float32)
    for _ in range(500):
        a, b = int(rng.integers(v)), int(rng.integers(v))
        if a == b:
            continue
        w = float(rng.integers(1, 1000))
        lines.append(f"{a} {b} {w}")
        x[a, b] = x[b, a] = np.float32(w)
    vmax = max(max(int(l.split()[0]), int(l.split()[1])) for l in lines[1:])
    x = x[: vmax + 1, : vmax + 1]
    off = ~np.eye(vmax + 1, dtype=bool)
    x[off & (x == 0)] = FLT_MAX
    path = tmp_path / "g.pbbs"
    path.write_text("\n".join(lines) + "\n")
    it, got = run(app, ["mst", "-f", str(path)], tmp=str(tmp_path))
    want, it_want = oracle_closure("min_max", x, 1)
    assert it == it_want
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_bellman_ford_form(cuda, app, tmp_path):
    """--bf: X <- X (+) A0 (x) X with A0 the adjacency (the reference's APBF build)."""
    rng = np.random.default_rng(9)
    v = 100
    edges = [(int(rng.integers(v)), int(rng.integers(v)), float(rng.integers(1, 101))) for _ in range(300)]
    edges = [e for e in edges if e[0] != e[1]]
    a0 = np.full((v, v), FLT_MAX, np.float32)
    for a, b, w in edges:
        a0[a, b] = np.float32(w)
    np.fill_diagonal(a0, 0)
    it, got = run(app, ["apsp", "-f", "--bf"], stdin=edge_text(v, edges), tmp=str(tmp_path))
    x = a0.copy()
    it_want = 0
    while it_want < 500:
        it_want += 1
        xn = oracle.srgemm("min_plus", a0, x, x, do_epilogue=True)
        same = not np.any(np.abs(x.astype(np.float64) - xn) > 1e-4)
        x = xn
        if same:
            break
    assert it == it_want
    np.testing.assert_array_equal(got.view(np.uint32), x.view(np.uint32))
