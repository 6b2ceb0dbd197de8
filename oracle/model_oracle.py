"""CPU restatement of the learned result-count model (float64 NumPy).

TEST INFRASTRUCTURE ONLY: the checker of the device model in
gpu_self_join_b200/csrc/gsj_model.cu (forward pass, loss and gradient).  The
reference has no such model; this file restates the network the library
defines: 16 features -> 64 ReLU -> 32 ReLU -> 1, weights in one flat array
[W1 (64x16, row per hidden unit), b1 (64), W2 (32x64), b2 (32), W3 (32), b3].
The loss is the mean squared error of the output.
"""
from __future__ import annotations

import numpy as np

F, H1, H2 = 16, 64, 32
NW = H1 * F + H1 + H2 * H1 + H2 + H2 + 1


def unpack(w: np.ndarray):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + H1 * F].reshape(H1, F); o += H1 * F
    b1 = w[o:o + H1]; o += H1
    W2 = w[o:o + H2 * H1].reshape(H2, H1); o += H2 * H1
    b2 = w[o:o + H2]; o += H2
    W3 = w[o:o + H2]; o += H2
    b3 = w[o]
    return W1, b1, W2, b2, W3, b3


def forward(w: np.ndarray, X: np.ndarray) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.maximum(X.astype(np.float64) @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3 + b3


def loss_grad(w: np.ndarray, X: np.ndarray, y: np.ndarray):
    """(mean squared error, gradient[NW]) in float64."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    X = X.astype(np.float64)
    n = X.shape[0]
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    out = h2 @ W3 + b3
    r = out - y.astype(np.float64)
    loss = float(np.mean(r * r))
    g = 2.0 * r / n
    dW3 = h2.T @ g
    db3 = g.sum()
    d2 = np.outer(g, W3) * (a2 > 0)
    dW2 = d2.T @ h1
    db2 = d2.sum(0)
    d1 = (d2 @ W2) * (a1 > 0)
    dW1 = d1.T @ X
    db1 = d1.sum(0)
    grad = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3, [db3]])
    return loss, grad
