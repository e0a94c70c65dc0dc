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
