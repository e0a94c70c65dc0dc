"""Train the learned-dispatch cost model and write costmodel_weights.json.

    python -m simd2_b200.train_costmodel [--out PATH] [--steps N]

Profiles min_plus closures of a fixed set of seeded R-MAT and Erdos-Renyi
graphs (n 512..4096, average degree 2..512) under all eight kernel
configurations (autotune.profile_closure), trains the MLP on the GPU with
libsimd2's own kernels, and stores the weights plus a summary of the
training data next to this file.  The dispatcher (simd2_closure_ex with
dispatch="learned") takes these weights.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import torch

from . import autotune, costmodel, datagen

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "costmodel_weights.json")

TRAIN_SET = ([("rmat", n, d) for n in (512, 1024, 2048, 4096) for d in (2, 4, 16, 64, 512)]
             + [("er", n, p) for n in (1024, 4096) for p in (0.001, 0.01)])


def make_graph(kind, n, param, seed):
    if kind == "rmat":
        return datagen.rmat_graph(n, float(param), seed=seed)
    return datagen.er_graph(n, float(param), seed=seed)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--records", default=None, help="also save the raw autotuner records here")
    args = ap.parse_args()
    dev = torch.device("cuda")
    t0 = time.time()
    recs = []
    for i, (kind, n, param) in enumerate(TRAIN_SET):
        g = torch.from_numpy(make_graph(kind, n, param, seed=1000 + i)).to(dev)
        recs.append(autotune.profile_closure("min_plus", g))
    if args.records:
        autotune.save(recs, args.records)
    X, y = autotune.dataset(recs)
    params, losses = costmodel.train(X.to(dev), y.to(dev), steps=args.steps, lr=3e-3)
    costmodel.save(params, args.out)
    summary = {"graphs": len(recs), "rows": int(X.shape[0]), "loss_first": losses[0], "loss_last": losses[-1],
               "best_fixed": autotune.describe(recs), "seconds": round(time.time() - t0, 1)}
    with open(args.out) as f:
        d = json.load(f)
    d["training"] = summary
    with open(args.out, "w") as f:
        json.dump(d, f)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
