"""Learned cost model of the closure-step dispatch.

A 15-32-32-1 ReLU MLP predicts log2(device time in ms) of one closure step
for each of the eight dense kernel configurations (split-K 1/2/4/8 x block
skip) and for a CSR SpGEMM step (configuration 8), from nine features of the
step's matrix: its block occupancy, stored entries and the products a sparse
step would form (``simd2_closure_ex`` computes them on the device).  Training and inference run on the GPU through
libsimd2's own kernels (``simd2_mlp_forward``, ``simd2_mlp_gradient`` with a
deterministic batch sum, ``simd2_mlp_adam``); the dispatcher evaluates the
network inside ``simd2_closure_ex`` (dispatch="learned").
"""
from __future__ import annotations

import ctypes
import json
import math

import numpy as np
import torch

from . import _check, _stream, lib

N_IN = 15
N_FEAT = 9
SPARSE = 8
HIDDEN = 32


def param_count() -> int:
    return int(lib().simd2_mlp_param_count())


def init_params(seed: int = 0, device="cuda") -> torch.Tensor:
    """He-style initialisation, flat layout W1|b1|W2|b2|W3|b3."""
    g = np.random.default_rng(seed)
    w1 = g.standard_normal((HIDDEN, N_IN)) * math.sqrt(2.0 / N_IN)
    w2 = g.standard_normal((HIDDEN, HIDDEN)) * math.sqrt(2.0 / HIDDEN)
    w3 = g.standard_normal(HIDDEN) * math.sqrt(1.0 / HIDDEN)
    flat = np.concatenate([w1.ravel(), np.zeros(HIDDEN), w2.ravel(), np.zeros(HIDDEN), w3, [0.0]]).astype(np.float32)
    assert flat.size == param_count()
    return torch.from_numpy(flat).to(device)


def encode(features, config: int) -> list:
    """Cost-model input: step features + one-hot split + skip flag + sparse flag."""
    if config == SPARSE:
        return list(features) + [0.0] * 5 + [1.0]
    s = config & 3
    return list(features) + [1.0 if j == s else 0.0 for j in range(4)] + [float(config >> 2), 0.0]


def forward(params: torch.Tensor, X: torch.Tensor, stream=None) -> torch.Tensor:
    X = X.contiguous().float()
    out = torch.empty(X.shape[0], dtype=torch.float32, device=X.device)
    _check(lib().simd2_mlp_forward(params.data_ptr(), X.data_ptr(), X.shape[0], out.data_ptr(), _stream(stream)),
           "mlp_forward")
    return out


def gradient(params: torch.Tensor, X: torch.Tensor, y: torch.Tensor, stream=None) -> torch.Tensor:
    X = X.contiguous().float()
    y = y.contiguous().float()
    P = param_count()
    grad = torch.empty(P, dtype=torch.float32, device=X.device)
    scratch = torch.empty((X.shape[0], P), dtype=torch.float32, device=X.device)
    _check(lib().simd2_mlp_gradient(params.data_ptr(), X.data_ptr(), y.data_ptr(), X.shape[0], grad.data_ptr(),
                                    scratch.data_ptr(), _stream(stream)), "mlp_gradient")
    return grad


def train(X: torch.Tensor, y: torch.Tensor, steps: int = 2000, lr: float = 3e-3, seed: int = 0,
          params: torch.Tensor | None = None):
    """Full-batch Adam on the GPU kernels; returns (params, loss history)."""
    X = X.contiguous().float()
    y = y.contiguous().float()
    P = param_count()
    params = init_params(seed, X.device) if params is None else params.clone()
    m = torch.zeros(P, device=X.device)
    v = torch.zeros(P, device=X.device)
    grad = torch.empty(P, dtype=torch.float32, device=X.device)
    scratch = torch.empty((X.shape[0], P), dtype=torch.float32, device=X.device)
    s = _stream(None)
    losses = []
    for t in range(1, steps + 1):
        _check(lib().simd2_mlp_gradient(params.data_ptr(), X.data_ptr(), y.data_ptr(), X.shape[0], grad.data_ptr(),
                                        scratch.data_ptr(), s), "mlp_gradient")
        _check(lib().simd2_mlp_adam(params.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(),
                                    ctypes.c_float(lr), t, s), "mlp_adam")
        if t == 1 or t % 100 == 0 or t == steps:
            losses.append(float(((forward(params, X) - y) ** 2).mean()))
    return params, losses


def save(params: torch.Tensor, path: str):
    with open(path, "w") as f:
        json.dump({"hidden": HIDDEN, "inputs": N_IN, "params": params.cpu().tolist()}, f)


def load_dense_table(path: str):
    """The autotuner's dense split table stored with the weights ([] if none)."""
    with open(path) as f:
        return [tuple(x) for x in json.load(f).get("training", {}).get("dense_configs", [])]


def load(path: str, device="cuda") -> torch.Tensor:
    """Weights saved by ``save``; raises unless they fit this network (the
    dispatcher reads simd2_mlp_param_count() floats from the array)."""
    with open(path) as f:
        d = json.load(f)
    if d.get("inputs") != N_IN or d.get("hidden") != HIDDEN or len(d["params"]) != param_count():
        raise ValueError(f"{path}: weights of a {d.get('inputs')}-input network with {len(d['params'])} parameters, "
                         f"not the {N_IN}-input network with {param_count()}")
    return torch.tensor(d["params"], dtype=torch.float32, device=device)
