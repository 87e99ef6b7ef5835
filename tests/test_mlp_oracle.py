"""The numpy checker of the surrogate network (oracle/mlp_oracle.py) pinned
by finite differences -- no GPU needed."""

import numpy as np

from oracle import mlp_oracle


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mlp_oracle.P)
    x = rng.uniform(-1, 1, 12)
    t = np.sin(2 * x)
    loss, g = mlp_oracle.loss_grad(p, x, t)
    idx = rng.choice(mlp_oracle.P, 60, replace=False)
    for i in idx:
        e = np.zeros(mlp_oracle.P)
        e[i] = 1e-6
        fd = (mlp_oracle.loss_grad(p + e, x, t)[0] -
              mlp_oracle.loss_grad(p - e, x, t)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i]))
    assert abs(loss - np.mean((mlp_oracle.forward(p, x) - t) ** 2)) < 1e-14


def test_adam_reduces_loss():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.2, mlp_oracle.P)
    x = np.linspace(-1, 1, 20)
    t = np.tanh(3 * x)
    p2, m, v, losses = mlp_oracle.adam(p, x, t, 300, 3e-3)
    assert losses[-1] < 0.05 * losses[0]
