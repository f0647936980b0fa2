"""Pins the numpy MLP oracle (oracle/mlp.py) by central finite differences."""
import numpy as np

from oracle import mlp


def test_mlp_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n = mlp.F * mlp.H + mlp.H + mlp.H * mlp.H + mlp.H + mlp.H * mlp.O + mlp.O
    p = rng.standard_normal(n) * 0.1
    X = rng.standard_normal((8, mlp.F))
    T = rng.standard_normal((8, mlp.O))
    loss, g, _ = mlp.loss_and_grads(p, X, T)
    h = 1e-6
    for i in rng.choice(n, 40, replace=False):
        e = np.zeros(n)
        e[i] = h
        fd = (mlp.loss_and_grads(p + e, X, T)[0] - mlp.loss_and_grads(p - e, X, T)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i]))
