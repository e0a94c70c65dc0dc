"""Train the learned-dispatch cost model and write costmodel_weights.json.

    python -m simd2_b200.train_costmodel [--out PATH] [--steps N]

Profiles min_plus closures of a fixed set of seeded R-MAT and Erdos-Renyi
graphs (n 2048..16384, average degree 2..2048) under all eight dense kernel
configurations and the sparse (CSR SpGEMM) configuration
(autotune.profile_closure), trains the MLP on the GPU with libsimd2's own
kernels, and stores the weights plus a summary of the training data next to
this file.  The dispatcher (simd2_closure_ex with dispatch="learned") takes
these weights; the summary's best fixed dense configuration is the one the
hand-written rules policy (dispatch="rules") runs.  The graphs are drawn
with other seeds than the mixed-density benchmark set.
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

TRAIN_SET = ([("rmat", n, d) for n in (2048, 4096) for d in (2, 4, 16, 64, 512)]
             + [("rmat", 8192, d) for d in (3, 8, 24, 96, 1024)]
             + [("rmat", 16384, d) for d in (4, 20, 300)]
             + [("er", 4096, 0.001), ("er", 8192, 0.0005)])


def make_graph(kind, n, param, seed, dev):
    if kind == "rmat":
        return datagen.rmat_graph_device(n, float(param), seed=seed, device=dev)
    return torch.from_numpy(datagen.er_graph(n, float(param), seed=seed)).to(dev)


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
        g = make_graph(kind, n, param, seed=1000 + i, dev=dev)
        recs.append(autotune.profile_closure("min_plus", g))
        del g
    if args.records:
        autotune.save(recs, args.records)
    X, y = autotune.dataset(recs)
    params, losses = costmodel.train(X.to(dev), y.to(dev), steps=args.steps, lr=3e-3)
    costmodel.save(params, args.out)
    summary = {"graphs": len(recs), "rows": int(X.shape[0]), "loss_first": losses[0], "loss_last": losses[-1],
               "best_fixed": autotune.describe(recs), "best_fixed_config": int(autotune.best_fixed(recs)[0]),
               "dense_configs": autotune.dense_table(recs),
               "seconds": round(time.time() - t0, 1)}
    with open(args.out) as f:
        d = json.load(f)
    d["training"] = summary
    with open(args.out, "w") as f:
        json.dump(d, f)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
