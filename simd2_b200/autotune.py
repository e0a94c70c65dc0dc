"""Autotuner of the closure-step kernel configuration.

Runs a closure once per configuration (split-K 1/2/4/8 x block skip, and
the sparse configuration: CSR SpGEMM steps while X is sparse) with
``simd2_closure_ex(dispatch="fixed")`` and records, for every step, the
cost-model features and each configuration's device time.  Every
configuration computes the same bits, so step t of all runs sees the same
matrix.  The records train the cost model (``costmodel.train``) and give the
best fixed configuration per workload; they are cached as JSON.
"""
from __future__ import annotations

import json
import math

import torch

from . import NUM_CONFIGS, SPARSE_CONFIG, closure_ex, config_desc


_warm = set()


def warm_up(op: str, device) -> None:
    """Loads every configuration's kernel once so no timing includes module loading."""
    if (op, str(device)) in _warm:
        return
    from .datagen import rmat_graph
    g = torch.from_numpy(rmat_graph(256, 4.0, seed=0)).to(device)
    for cfg in range(NUM_CONFIGS + 1):
        closure_ex(op, g.clone(), dispatch="fixed", config=cfg)
    _warm.add((op, str(device)))


def profile_closure(op: str, X0: torch.Tensor, configs=range(NUM_CONFIGS + 1), repeats: int = 1,
                    max_iter: int = 500):
    """Per-step timings of every configuration on one input matrix.

    Returns {"n", "iters", "features": [step][9], "ms": {config: [step]}};
    the sparse configuration's list holds None for the steps it did not run
    sparse (X too dense for the sparse store, or past n^3/16 products).
    """
    warm_up(op, X0.device)
    rec = {"n": int(X0.shape[0]), "ms": {}}
    for cfg in configs:
        best = None
        for _ in range(repeats):
            X = X0.clone()
            r = closure_ex(op, X, dispatch="fixed", config=cfg, max_iter=max_iter, record=True)
            ms = r["ms"]
            if cfg == SPARSE_CONFIG:
                ms = [m if c == SPARSE_CONFIG else None for m, c in zip(r["ms"], r["configs"])]
            best = ms if best is None else [None if a is None else min(a, b) for a, b in zip(best, ms)]
            rec["iters"] = r["iters"]
            if cfg != SPARSE_CONFIG:
                rec["features"] = r["features"]
        rec["ms"][int(cfg)] = best
    return rec


def dataset(records):
    """(inputs [rows][15], targets log2(ms) [rows]) from profile records."""
    from .costmodel import encode
    xs, ys = [], []
    for rec in records:
        for cfg, times in rec["ms"].items():
            for t, ms in enumerate(times):
                if ms is None:
                    continue
                xs.append(encode(rec["features"][t], int(cfg)))
                ys.append(math.log2(max(ms, 1e-4)))
    return torch.tensor(xs, dtype=torch.float32), torch.tensor(ys, dtype=torch.float32)


def best_fixed(records):
    """Dense configuration with the smallest total time over all records."""
    tot = {}
    for rec in records:
        for cfg, times in rec["ms"].items():
            if int(cfg) < NUM_CONFIGS:
                tot[int(cfg)] = tot.get(int(cfg), 0.0) + sum(times)
    return min(tot, key=tot.get), tot


def dense_table(records):
    """The plain dense path's split-K factor by size: for every n profiled, the
    configuration without block skipping (split 1/2/4/8) with the smallest
    total time over that n's records, as [(n, config)] ascending in n
    (``simd2_b200.set_dense_configs`` installs it)."""
    tot = {}
    for rec in records:
        for cfg in range(4):
            t = tot.setdefault(int(rec["n"]), {})
            t[cfg] = t.get(cfg, 0.0) + sum(rec["ms"][cfg])
    return [(n, min(t, key=t.get)) for n, t in sorted(tot.items())]


def save(records, path):
    with open(path, "w") as f:
        json.dump(records, f)


def load(path):
    with open(path) as f:
        recs = json.load(f)
    for r in recs:
        r["ms"] = {int(k): v for k, v in r["ms"].items()}
    return recs


def describe(records):
    cfg, tot = best_fixed(records)
    return {config_desc(c): round(t, 3) for c, t in sorted(tot.items())} | {"best": config_desc(cfg)}
