"""CPU oracle of the learned initial-guess MLP (test infrastructure only).

FP64 numpy restatement of the per-sample network out = w2 . relu(W1 x + b1) +
b2 and of the gradient of the mean squared error L = mean((out - y)^2), with
the parameter layout of the device implementation: W1 (H x D, row-major), b1
(H), w2 (H), b2 (1). Used to check the device kernels' forward values and
gradients; pinned itself by central finite differences in the CPU tests.
(The network has no reference counterpart; the restatement follows the
standard back-propagation of a two-layer ReLU network.)
"""
from __future__ import annotations

import numpy as np


def unpack(p, D, H):
    p = np.asarray(p, dtype=np.float64)
    W1 = p[: H * D].reshape(H, D)
    b1 = p[H * D: H * D + H]
    w2 = p[H * D + H: H * D + 2 * H]
    b2 = p[H * D + 2 * H]
    return W1, b1, w2, b2


def forward(p, X, D, H):
    W1, b1, w2, b2 = unpack(p, D, H)
    A = np.asarray(X, dtype=np.float64) @ W1.T + b1
    return np.maximum(A, 0.0) @ w2 + b2


def loss_and_grad(p, X, y, D, H):
    W1, b1, w2, b2 = unpack(p, D, H)
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    m = X.shape[0]
    A = X @ W1.T + b1
    Hh = np.maximum(A, 0.0)
    out = Hh @ w2 + b2
    e = out - y
    loss = float(np.mean(e * e))
    g = 2.0 * e / m
    gw2 = Hh.T @ g
    gb2 = g.sum()
    GH = np.outer(g, w2) * (A > 0)
    gW1 = GH.T @ X
    gb1 = GH.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gw2, [gb2]])
