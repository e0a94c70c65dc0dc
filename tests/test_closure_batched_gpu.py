"""Batched closure (one persistent launch) against the oracle, graph by graph."""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu


def bits(x):
    return np.ascontiguousarray(x).view(np.uint32)


@pytest.mark.parametrize("op", ["min_plus", "max_min", "min_max", "max_mul"])
def test_batched_matches_oracle(cuda, op):
    rng = np.random.default_rng(11)
    sizes = [1, 2, 3, 31, 32, 33, 64, 127, 128, 129, 200, 255, 257, 300] + list(rng.integers(1, 260, 10))
    graphs = []
    for i, n in enumerate(sizes):
        if op == "max_mul":  # reliability-style weights in (0,1], diag 1
            x = rng.random((n, n)).astype(np.float32)
            x[rng.random((n, n)) > 0.1] = 0.0
            np.fill_diagonal(x, 1.0)
            graphs.append(x.astype(np.float32))
        else:
            graphs.append(datagen.closure_graph(op if op != "min_max" else "min_plus", int(n),
                                                float(rng.uniform(0.01, 0.3)), seed=i))
    mats = [torch.from_numpy(g.copy()).to(cuda) for g in graphs]
    iters = s2.closure_batched(op, mats)
    for g, m, it in zip(graphs, mats, iters):
        want, it_want = oracle.closure(op, g)
        assert it == it_want, (g.shape, it, it_want)
        np.testing.assert_array_equal(bits(m.cpu().numpy()), bits(want), err_msg=f"n={g.shape[0]}")
    assert s2.device_status() == 0


def test_batched_strided_views_and_plan_replay(cuda):
    """Row pitch > n, and a plan run twice on restored inputs gives the same answer."""
    rng = np.random.default_rng(5)
    sizes = [50, 130, 7]
    graphs = [datagen.er_graph(n, 0.1, seed=n) for n in sizes]
    bigs = [torch.full((n, n + 9), 3.0, device=cuda) for n in sizes]
    for b, g in zip(bigs, graphs):
        b[:, : g.shape[0]] = torch.from_numpy(g).to(cuda)
    views = [b[:, : g.shape[0]] for b, g in zip(bigs, graphs)]
    plan = s2.BatchedClosure("min_plus", views)
    for rep in range(2):
        for b, g in zip(bigs, graphs):
            b[:, : g.shape[0]] = torch.from_numpy(g).to(cuda)
        plan.run()
        torch.cuda.synchronize()
        its, nc = plan.iters()
        assert nc == 0
        for v, b, g, it in zip(views, bigs, graphs, its):
            want, it_want = oracle.closure("min_plus", g)
            assert it == it_want
            np.testing.assert_array_equal(bits(v.cpu().numpy()), bits(want))
            assert torch.all(b[:, g.shape[0]:] == 3.0)
    plan.close()


def test_batched_cuda_graph_capture(cuda):
    graphs = [datagen.er_graph(n, 0.05, seed=n) for n in (90, 40, 200)]
    mats = [torch.from_numpy(g.copy()).to(cuda) for g in graphs]
    plan = s2.BatchedClosure("min_plus", mats)
    s = torch.cuda.Stream()
    plan.run(stream=s)  # warm-up outside capture (module load, attributes)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.run(stream=s)
    for m, x in zip(mats, graphs):
        m.copy_(torch.from_numpy(x))
    g.replay()
    torch.cuda.synchronize()
    for m, x in zip(mats, graphs):
        want, _ = oracle.closure("min_plus", x)
        np.testing.assert_array_equal(bits(m.cpu().numpy()), bits(want))
    del g
    plan.close()


def test_batched_not_converged_and_empty(cuda):
    n = 40
    x = np.full((n, n), np.inf, np.float32)
    np.fill_diagonal(x, 0)
    for i in range(n - 1):
        x[i, i + 1] = 1.0
    m = torch.from_numpy(x).to(cuda)
    with pytest.raises(s2.NotConverged):
        s2.closure_batched("min_plus", [m], max_iter=2)
    assert s2.closure_batched("min_plus", []) == []


@pytest.mark.parametrize("op", ["max_min", "min_max"])
@pytest.mark.parametrize("case", ["fp16", "one-off", "overflow", "tol"])
def test_batched_selection_fp16_and_fp32_paths(cuda, op, case):
    """max_min / min_max close every graph on FP16 copies when every entry of
    every graph is an FP16 value (integer weights), else on FP32: one entry
    that is not (1.0001, or 70000 past the FP16 range) sends the whole batch
    to FP32.  Same bits and step counts as the oracle either way, under the
    bitwise and the |delta| > 1e-4 change tests; also replayed from a
    captured CUDA graph."""
    rng = np.random.default_rng(17)
    sizes = [5, 64, 65, 127, 128, 129, 191, 200, 256, 300, 33, 1]
    graphs = [datagen.closure_graph(op if op == "max_min" else "min_plus", int(n), float(rng.uniform(0.02, 0.3)),
                                    seed=40 + i) for i, n in enumerate(sizes)]
    if case == "one-off":
        graphs[3][5, 7] = np.float32(1.0001)
    elif case == "overflow":
        graphs[7][2, 3] = np.float32(70000.0)
    conv = "tol" if case == "tol" else "exact"
    mats = [torch.from_numpy(g.copy()).to(cuda) for g in graphs]
    plan = s2.BatchedClosure(op, mats, conv=conv)
    s = torch.cuda.Stream()
    plan.run(stream=s)
    s.synchronize()
    for rep in range(2):
        if rep == 1:  # the second run replays a captured CUDA graph on restored inputs
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg, stream=s):
                plan.run(stream=s)
            for m, g in zip(mats, graphs):
                m.copy_(torch.from_numpy(g))
            cg.replay()
            torch.cuda.synchronize()
        its, nc = plan.iters()
        assert nc == 0
        for g, m, it in zip(graphs, mats, its):
            want, it_want = oracle.closure(op, g, tol_mode=1 if conv == "tol" else 0)
            assert it == it_want, (case, g.shape, it, it_want)
            np.testing.assert_array_equal(bits(m.cpu().numpy()), bits(want), err_msg=f"{case} n={g.shape[0]}")
        if rep == 1:
            del cg
    plan.close()
    assert s2.device_status() == 0
