"""Kernel configurations (split-K clusters, block skipping) and the learned dispatch."""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from oracle import mlp as mlp_oracle
from simd2_b200 import autotune, costmodel, datagen

pytestmark = pytest.mark.gpu
SKIPPABLE = ["min_plus", "max_plus", "max_min", "min_max"]


def bits(x):
    return np.ascontiguousarray(x).view(np.uint32)


def sparse_operands(op, m, n, k, seed, density):
    """Operands whose blocks are often entirely the (x)-annihilator."""
    a, b, c = datagen.semiring_operands(op, m, n, k, seed=seed)
    ann = np.float32(np.inf if op in ("min_plus", "min_max", "min_mul") else -np.inf)
    rng = np.random.default_rng(seed)
    # zero out whole 32 x 32 blocks with probability 1 - density
    for x in (a, b):
        br, bc = (x.shape[0] + 31) // 32, (x.shape[1] + 31) // 32
        keep = rng.random((br, bc)) < density
        mask = np.repeat(np.repeat(keep, 32, 0), 32, 1)[: x.shape[0], : x.shape[1]]
        x[~mask] = ann
    return a, b, c


@pytest.mark.parametrize("op", SKIPPABLE + ["max_mul", "min_mul"])
@pytest.mark.parametrize("shape", [(300, 260, 517), (128, 128, 96), (1, 513, 33), (700, 130, 1024)])
def test_all_configs_bit_exact(cuda, op, shape):
    m, n, k = shape
    a, b, c = sparse_operands(op, m, n, k, seed=m + k, density=0.3)
    want = oracle.srgemm(op, a, b, c, do_epilogue=True)
    A, B, C = (torch.from_numpy(x).to(cuda) for x in (a, b, c))
    for cfg in range(s2.NUM_CONFIGS):
        D = s2.srgemm_tuned(op, A, B, C, do_epilogue=True, config=cfg)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(bits(D.cpu().numpy()), bits(want), err_msg=f"{op} {shape} {s2.config_desc(cfg)}")
    assert s2.device_status() == 0


def test_empty_k_lists(cuda):
    """Rows/columns made only of +inf: every k-block is skipped, D = C."""
    a = np.full((256, 300), np.inf, np.float32)
    b = np.full((300, 256), np.inf, np.float32)
    c = np.random.default_rng(1).random((256, 256)).astype(np.float32)
    A, B, C = (torch.from_numpy(x).to(cuda) for x in (a, b, c))
    for cfg in (4, 5, 7):
        D = s2.srgemm_tuned("min_plus", A, B, C, do_epilogue=True, config=cfg)
        np.testing.assert_array_equal(D.cpu().numpy(), c)


@pytest.mark.parametrize("op", ["min_plus", "max_min"])
def test_closure_every_config_identical(cuda, op):
    x = datagen.rmat_graph(512, 3.0, seed=4) if op == "min_plus" else datagen.closure_graph(op, 400, 0.01, seed=4)
    want, it_want = oracle.closure(op, x)
    for cfg in range(s2.NUM_CONFIGS):
        X = torch.from_numpy(x.copy()).to(cuda)
        r = s2.closure_ex(op, X, dispatch="fixed", config=cfg, record=True)
        assert r["iters"] == it_want
        np.testing.assert_array_equal(bits(X.cpu().numpy()), bits(want), err_msg=s2.config_desc(cfg))
        assert all(c == cfg for c in r["configs"])


def test_mlp_gradient_matches_fp64_oracle(cuda):
    rng = np.random.default_rng(3)
    p = (rng.standard_normal(costmodel.param_count()) * 0.3).astype(np.float32)
    X = rng.standard_normal((97, costmodel.N_IN)).astype(np.float32)
    y = rng.standard_normal(97).astype(np.float32)
    P = torch.from_numpy(p).to(cuda)
    g = costmodel.gradient(P, torch.from_numpy(X).to(cuda), torch.from_numpy(y).to(cuda)).cpu().numpy()
    want = mlp_oracle.gradient(p.astype(np.float64), X.astype(np.float64), y.astype(np.float64))
    scale = np.abs(want).max()
    np.testing.assert_allclose(g, want, rtol=1e-3, atol=1e-5 * scale)
    out = costmodel.forward(P, torch.from_numpy(X).to(cuda)).cpu().numpy()
    np.testing.assert_allclose(out, mlp_oracle.forward(p.astype(np.float64), X.astype(np.float64))[0], rtol=1e-4,
                               atol=1e-5)
    # deterministic batch sum: same gradient bits twice
    g2 = costmodel.gradient(P, torch.from_numpy(X).to(cuda), torch.from_numpy(y).to(cuda)).cpu().numpy()
    np.testing.assert_array_equal(g, g2)


def test_mlp_training_fits(cuda):
    rng = np.random.default_rng(5)
    X = rng.random((512, costmodel.N_IN)).astype(np.float32)
    y = (np.sin(3 * X[:, 0]) + X[:, 1] * X[:, 2] - X[:, 7]).astype(np.float32)
    Xt, yt = torch.from_numpy(X).to(cuda), torch.from_numpy(y).to(cuda)
    params, losses = costmodel.train(Xt, yt, steps=1500, lr=3e-3)
    assert losses[-1] < 0.1 * losses[0]
    assert losses[-1] < 0.01


def test_learned_dispatch_identical_and_not_slower(cuda):
    """Train on autotuner timings of some R-MAT closures (every dense
    configuration and the sparse one), then close held-out R-MAT graphs with
    the dense path, the rules policy and the learned dispatch: the same bits
    and step counts, and the learned dispatch no slower than the dense path."""
    train_graphs = [datagen.rmat_graph(2048, d, seed=10 + i) for i, d in enumerate((2, 8, 64))]
    recs = [autotune.profile_closure("min_plus", torch.from_numpy(g).to(cuda)) for g in train_graphs]
    assert any(m is not None for r in recs for m in r["ms"][s2.SPARSE_CONFIG])
    Xd, yd = autotune.dataset(recs)
    assert Xd.shape[1] == costmodel.N_IN
    params, losses = costmodel.train(Xd.to(cuda), yd.to(cuda), steps=1500)
    assert losses[-1] < losses[0]
    t_dense = t_learned = 0.0
    for i, d in enumerate((3, 16)):
        g = datagen.rmat_graph(4096, d, seed=100 + i)
        Xa = torch.from_numpy(g.copy()).to(cuda)
        Xb = torch.from_numpy(g.copy()).to(cuda)
        Xc = torch.from_numpy(g.copy()).to(cuda)
        ra = s2.closure_ex("min_plus", Xa, dispatch="dense", record=True)
        rb = s2.closure_ex("min_plus", Xb, dispatch="learned", mlp_params=params, record=True)
        rc = s2.closure_ex("min_plus", Xc, dispatch="rules", config=s2.config_id(2, True), record=True)
        assert ra["iters"] == rb["iters"] == rc["iters"]
        assert torch.equal(Xa.view(torch.int32), Xb.view(torch.int32))
        assert torch.equal(Xa.view(torch.int32), Xc.view(torch.int32))
        t_dense += sum(ra["ms"])
        t_learned += sum(rb["ms"])
    assert t_learned <= 1.05 * t_dense, (t_learned, t_dense)


def test_fixed_sparse_config_records_sparse_steps(cuda):
    """dispatch="fixed" with the sparse configuration: CSR SpGEMM steps while
    X fits the sparse store, then the dense path; same bits and steps as the
    dense path, and a time recorded for every sparse step."""
    x = datagen.rmat_graph(2048, 4.0, seed=41)
    Xa = torch.from_numpy(x.copy()).to(cuda)
    Xb = torch.from_numpy(x.copy()).to(cuda)
    ra = s2.closure_ex("min_plus", Xa, dispatch="dense", record=True)
    rb = s2.closure_ex("min_plus", Xb, dispatch="fixed", config=s2.SPARSE_CONFIG, record=True)
    assert ra["iters"] == rb["iters"]
    assert torch.equal(Xa.view(torch.int32), Xb.view(torch.int32))
    assert rb["configs"][0] == s2.SPARSE_CONFIG
    assert all(m > 0 for m, c in zip(rb["ms"], rb["configs"]) if c == s2.SPARSE_CONFIG)


def test_learned_dispatch_small_closure_runs_dense_path(cuda):
    """At n <= 1024 a per-step decision costs about a dense step, so the learned
    policy runs the plain path: same bits, same per-step configurations, no
    features recorded."""
    params = torch.randn(costmodel.param_count(), generator=torch.Generator().manual_seed(0)).to(cuda)
    x = datagen.er_graph(512, 0.05, seed=1)
    want, it_want = oracle.closure("min_plus", x)
    Xa = torch.from_numpy(x.copy()).to(cuda)
    Xb = torch.from_numpy(x.copy()).to(cuda)
    ra = s2.closure_ex("min_plus", Xa, dispatch="dense", record=True)
    rb = s2.closure_ex("min_plus", Xb, dispatch="learned", mlp_params=params, record=True)
    assert ra["iters"] == rb["iters"] == it_want
    assert ra["configs"] == rb["configs"]
    assert all(f == [0.0] * costmodel.N_FEAT for f in rb["features"])
    np.testing.assert_array_equal(bits(Xb.cpu().numpy()), bits(want))


@pytest.mark.parametrize("case", ["rmat", "components"])
def test_learned_sparse_opening_identical(cuda, case):
    """Above n = 1024 the rules and learned policies may square a sparse X as
    CSR SpGEMM steps (config 8) before the dense steps: same bits and the same
    step count as the dense path, whatever an (untrained) MLP chooses.
    'components' (disjoint 4-cycles) converges while still sparse."""
    n = 2048
    if case == "rmat":
        x = datagen.rmat_graph(n, 3.0, seed=21)
    else:
        rng = np.random.default_rng(22)
        x = np.full((n, n), np.inf, np.float32)
        np.fill_diagonal(x, 0.0)
        for b in range(0, n, 4):
            for t in range(4):
                x[b + t, b + (t + 1) % 4] = rng.integers(1, 100)
    Xa = torch.from_numpy(x.copy()).to(cuda)
    ra = s2.closure_ex("min_plus", Xa, dispatch="dense", record=True)
    Xr = torch.from_numpy(x.copy()).to(cuda)
    rr = s2.closure_ex("min_plus", Xr, dispatch="rules", config=s2.config_id(2, True), record=True)
    assert rr["iters"] == ra["iters"]
    assert torch.equal(Xa.view(torch.int32), Xr.view(torch.int32))
    assert rr["configs"][0] == s2.SPARSE_CONFIG  # the rules' opening ran
    if case == "components":
        assert all(c == s2.SPARSE_CONFIG for c in rr["configs"])
    for seed in (1, 2, 3):
        params = torch.randn(costmodel.param_count(), generator=torch.Generator().manual_seed(seed)).to(cuda)
        Xb = torch.from_numpy(x.copy()).to(cuda)
        rb = s2.closure_ex("min_plus", Xb, dispatch="learned", mlp_params=params, record=True)
        assert rb["iters"] == ra["iters"]
        assert torch.equal(Xa.view(torch.int32), Xb.view(torch.int32))
        # without recording as well
        Xc = torch.from_numpy(x.copy()).to(cuda)
        assert s2.closure_ex("min_plus", Xc, dispatch="learned", mlp_params=params) == ra["iters"]
        assert torch.equal(Xa.view(torch.int32), Xc.view(torch.int32))


@pytest.mark.parametrize("steps", [1, 2])
def test_learned_opening_step_cap(cuda, steps):
    """max_iter reached inside the sparse opening: NotConverged, and X holds
    exactly the dense path's X after the same number of squarings."""
    x = datagen.rmat_graph(4096, 4.0, seed=31)
    params = torch.randn(costmodel.param_count(), generator=torch.Generator().manual_seed(2)).to(cuda)
    Xa = torch.from_numpy(x.copy()).to(cuda)
    with pytest.raises(s2.NotConverged):
        s2.closure_ex("min_plus", Xa, dispatch="dense", max_iter=steps)
    for kw in ({"dispatch": "learned", "mlp_params": params}, {"dispatch": "rules", "config": 5},
               {"dispatch": "fixed", "config": s2.SPARSE_CONFIG}):
        Xb = torch.from_numpy(x.copy()).to(cuda)
        with pytest.raises(s2.NotConverged):
            s2.closure_ex("min_plus", Xb, max_iter=steps, **kw)
        assert torch.equal(Xa.view(torch.int32), Xb.view(torch.int32)), kw


def test_shipped_costmodel_on_held_out_graphs(cuda):
    """The shipped network (simd2_b200/costmodel_weights.json, trained on the
    GPU by the library's own kernels on autotuner timings) closes held-out
    R-MAT graphs -- seeds and degrees outside its training set -- with the
    dense path's bits and step counts, and against the method without it (the
    plain dense path, which takes no sparse steps and skips no blocks) it
    gains at least 1.1x.  Against the hand-written rules (sparse steps under
    fixed entry and product thresholds, then the autotuner's best fixed dense
    configuration), which it replaces, it must stay within 5 %: the best
    per-step choice on the training timings is within 1 % of those rules."""
    import json
    import os
    import time
    path = os.path.join(os.path.dirname(s2.__file__), "costmodel_weights.json")
    params = costmodel.load(path, cuda)
    with open(path) as f:
        rules_cfg = int(json.load(f)["training"]["best_fixed_config"])
    arms = {"dense": {"dispatch": "dense"}, "rules": {"dispatch": "rules", "config": rules_cfg},
            "learned": {"dispatch": "learned", "mlp_params": params}}
    graphs = [(4096, 6.0), (4096, 40.0), (4096, 300.0), (8192, 5.0), (8192, 50.0)]
    # warm-up: workspaces and kernels outside the timing
    for n in (4096, 8192):
        g = datagen.rmat_graph_device(n, 8.0, seed=1, device=cuda)
        for kw in arms.values():
            s2.closure_ex("min_plus", g.clone(), **kw)
    tot = {a: 0.0 for a in arms}
    for i, (n, d) in enumerate(graphs):
        g = datagen.rmat_graph_device(n, d, seed=7000 + i, device=cuda)
        out = {}
        for a, kw in arms.items():
            X = g.clone()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            it = s2.closure_ex("min_plus", X, **kw)
            tot[a] += time.perf_counter() - t0
            out[a] = (it, X)
        for a in ("rules", "learned"):
            assert out[a][0] == out["dense"][0]
            assert torch.equal(out[a][1].view(torch.int32), out["dense"][1].view(torch.int32)), (a, n, d)
    assert tot["dense"] >= 1.1 * tot["learned"], tot
    assert tot["learned"] <= 1.05 * tot["rules"], tot


def test_autotuned_dense_configs(cuda):
    """The plain dense path takes the split-K factor the autotuner installed
    for the closure's size (recorded per step), with the same bits as the
    rule's split; the shipped table is read from the weights file."""
    import os
    path = os.path.join(os.path.dirname(s2.__file__), "costmodel_weights.json")
    shipped = costmodel.load_dense_table(path)
    assert shipped and all(0 <= c <= 3 for _, c in shipped)
    x = datagen.rmat_graph(2048, 16.0, seed=61)
    Xa = torch.from_numpy(x.copy()).to(cuda)
    ra = s2.closure_ex("min_plus", Xa, dispatch="dense", record=True)
    assert all(c == 0 for c in ra["configs"])  # the rule: 256 tiles >= 148 SMs, split 1
    try:
        s2.set_dense_configs([(1024, 1), (4096, 2)])
        Xb = torch.from_numpy(x.copy()).to(cuda)
        rb = s2.closure_ex("min_plus", Xb, dispatch="dense", record=True)
        assert all(c == 1 for c in rb["configs"])  # n = 2048 falls in the entry from 1024: split 2
        assert rb["iters"] == ra["iters"]
        assert torch.equal(Xa.view(torch.int32), Xb.view(torch.int32))
        Xc = torch.from_numpy(x.copy()).to(cuda)
        assert s2.closure("min_plus", Xc) == ra["iters"]
        assert torch.equal(Xa.view(torch.int32), Xc.view(torch.int32))
    finally:
        s2.set_dense_configs([])
    Xd = torch.from_numpy(x.copy()).to(cuda)
    rd = s2.closure_ex("min_plus", Xd, dispatch="dense", record=True)
    assert rd["configs"] == ra["configs"]


@pytest.mark.parametrize("case", ["min_plus_rmat", "max_plus_dag"])
def test_delta_steps_identical(cuda, case):
    """The rules and learned loops of a min_plus / max_plus closure skip, from
    the second dense step on, the k-tiles whose A and B 32 x 32 blocks both
    stayed unchanged in the step before (their products are already folded in,
    so a min / max cannot change).  Unrecorded closures (recording keeps plain
    steps) must equal the plain dense closure bit for bit, with the same step
    count: an R-MAT graph for min_plus, and for max_plus (longest paths) a
    random DAG whose closure takes a dozen steps of shrinking change."""
    import os
    path = os.path.join(os.path.dirname(s2.__file__), "costmodel_weights.json")
    params = costmodel.load(path, cuda)
    if case == "min_plus_rmat":
        op, n = "min_plus", 4096
        g = datagen.rmat_graph_device(n, 70.0, seed=4242, device=cuda)
    else:
        op, n = "max_plus", 3072
        gen = torch.Generator(device=cuda).manual_seed(77)
        w = torch.randint(1, 101, (n, n), device=cuda, generator=gen).float()
        keep = (torch.rand((n, n), device=cuda, generator=gen) < 0.002) & torch.ones(n, n, device=cuda).triu(1).bool()
        g = torch.where(keep, w, torch.full_like(w, float("-inf")))
        g.fill_diagonal_(0.0)
    Xd = g.clone()
    it_d = s2.closure_ex(op, Xd, dispatch="dense")
    assert it_d >= 3
    for kw in ({"dispatch": "rules", "config": s2.config_id(1, True)}, {"dispatch": "learned", "mlp_params": params}):
        X = g.clone()
        it = s2.closure_ex(op, X, **kw)
        assert it == it_d, kw["dispatch"]
        assert torch.equal(X.view(torch.int32), Xd.view(torch.int32)), kw["dispatch"]
    assert s2.device_status() == 0
