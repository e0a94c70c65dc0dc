"""Row-panel closure on the GPU: the panel step (simd2_closure_panel_step)
and the exchange loop at one rank, against simd2_closure and the oracle.
The multi-rank exchange itself is covered on CPU (gloo) in test_shard_gloo;
here several ranks are emulated one after another on one GPU, each step
reading the same full X, so no kernel waits on another."""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen
from simd2_b200.shard import closure_rowpanel, panel_bounds

pytestmark = pytest.mark.gpu


def _bits(a):
    return a.view(np.uint8) if a.dtype == np.uint8 else a.view(np.uint32)


@pytest.mark.parametrize("op", ["min_plus", "max_min", "min_max"])
def test_single_rank_rowpanel_equals_closure(cuda, op):
    x = datagen.closure_graph(op, 300, 0.03, seed=11)
    X = torch.from_numpy(x).to(cuda)
    it = closure_rowpanel(op, X, 300)
    want, it_want = oracle.closure(op, x)
    assert it == it_want
    assert np.array_equal(_bits(X.cpu().numpy()), _bits(want))


@pytest.mark.parametrize("world", [2, 3, 5])
@pytest.mark.parametrize("op", ["min_plus", "or_and"])
def test_emulated_ranks_match_oracle(cuda, op, world):
    n = 257
    if op == "or_and":
        rng = np.random.default_rng(world)
        x = (rng.random((n, n)) < 0.01).astype(np.uint8)
        np.fill_diagonal(x, 1)
    else:
        x = datagen.er_graph(n, 0.02, seed=world)
    want, it_want = oracle.closure(op, x)
    P, bounds = panel_bounds(n, world)
    X = torch.from_numpy(x).to(cuda)
    changed = torch.zeros(1, dtype=torch.int32, device=cuda)
    it = 0
    while True:
        it += 1
        changed.zero_()
        new = torch.empty_like(X)
        for start, stop in bounds:  # one "rank" after another, all reading X_t
            if stop > start:
                s2.closure_panel_step(op, X[start:stop], X, new[start:stop], changed)
        X = new
        if changed.item() == 0 or it >= 500:
            break
    assert it == it_want
    assert np.array_equal(_bits(X.cpu().numpy()), _bits(want))


def test_panel_step_arguments(cuda):
    X = torch.zeros((64, 64), device=cuda)
    changed = torch.zeros(1, dtype=torch.int32, device=cuda)
    with pytest.raises(s2.Simd2Error):
        s2.closure_panel_step("min_plus", X[:32], X, X[:32], changed)  # out aliases panel
    with pytest.raises(TypeError):
        s2.closure_panel_step("or_and", X[:32], X, torch.empty_like(X[:32]), changed)
    with pytest.raises(ValueError):
        s2.closure_panel_step("min_plus", X[:32], X[:16], torch.empty_like(X[:32]), changed)
