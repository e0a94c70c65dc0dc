"""The FP64 MLP oracle against central finite differences (CPU)."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = 32 * mlp.N_IN + 32 + 32 * 32 + 32 + 32 + 1
    p = rng.standard_normal(P) * 0.3
    X = rng.standard_normal((9, mlp.N_IN))
    y = rng.standard_normal(9)

    def loss(q):
        out, _ = mlp.forward(q, X)
        return np.mean((out - y) ** 2)

    g = mlp.gradient(p, X, y)
    idx = rng.choice(P, size=60, replace=False)
    for i in idx:
        e = np.zeros(P)
        e[i] = 1e-6
        fd = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
