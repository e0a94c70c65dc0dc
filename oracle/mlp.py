"""FP64 CPU oracle of the cost-model MLP -- TEST INFRASTRUCTURE ONLY.

Restates the 15-32-32-1 ReLU network of simd2_b200/csrc/mlp.cuh (flat
parameter layout W1|b1|W2|b2|W3|b3) with its forward pass and the gradient of
mean((f(X) - y)^2), in float64, to check the GPU training kernels.
"""
import numpy as np

N_IN, H = 15, 32


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    w1 = p[o:o + H * N_IN].reshape(H, N_IN); o += H * N_IN
    b1 = p[o:o + H]; o += H
    w2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return w1, b1, w2, b2, w3, b3


def forward(p, X):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    z1 = X @ w1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ w3 + b3, (z1, h1, z2, h2)


def gradient(p, X, y):
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(p)
    out, (z1, h1, z2, h2) = forward(p, X)
    d = 2.0 * (out - y) / X.shape[0]
    gw3 = h2.T @ d
    gb3 = d.sum()
    d2 = (d[:, None] * w3[None, :]) * (z2 > 0)
    gw2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ w2) * (z1 > 0)
    gw1 = d1.T @ X
    gb1 = d1.sum(0)
    return np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2, gw3, [gb3]])
