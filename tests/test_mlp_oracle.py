"""The MLP oracle (oracle/mlp_oracle.py) pinned by central finite differences."""
from __future__ import annotations

import numpy as np

from oracle import mlp_oracle as MO


def test_mlp_oracle_gradient_matches_finite_differences():
    D, H, m = 5, 7, 40
    rng = np.random.default_rng(0)
    p = rng.standard_normal(H * D + 2 * H + 1) * 0.5
    X = rng.standard_normal((m, D))
    y = rng.standard_normal(m)
    loss, g = MO.loss_and_grad(p, X, y, D, H)
    assert np.isclose(loss, np.mean((MO.forward(p, X, D, H) - y) ** 2))
    h = 1e-6
    fd = np.empty_like(p)
    for k in range(p.size):
        dp = np.zeros_like(p)
        dp[k] = h
        fd[k] = (MO.loss_and_grad(p + dp, X, y, D, H)[0] - MO.loss_and_grad(p - dp, X, y, D, H)[0]) / (2 * h)
    assert np.abs(g - fd).max() <= 1e-6 * max(1.0, np.abs(fd).max())
