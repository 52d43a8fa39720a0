"""CPU restatement of the learned-boundary MLP (TEST INFRASTRUCTURE).

Only the test-suite uses this module, as the checker of the device kernels
(xfb_mlp_loss_grad / xfb_mlp_train): float64 forward and backward pass of
the network of csrc/labc.cuh with the weights rounded to BF16 (round to
nearest even) for the forward pass, as the kernels do; the gradient is taken
with respect to the rounded weights (straight-through rounding).
"""
from __future__ import annotations

import numpy as np

NI, NH = 8, 64
W1, B1 = 0, 8 * 64
W2 = B1 + 64
B2 = W2 + 64 * 64
W3 = B2 + 64
B3 = W3 + 64
NP = B3 + 1


def bf16(w: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    u = np.asarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    return (w[W1:B1].reshape(NH, NI), w[B1:W2], w[W2:B2].reshape(NH, NH), w[B2:W3], w[W3:B3], w[B3])


def loss_grad(x: np.ndarray, y: np.ndarray, w: np.ndarray):
    """Mean squared error and its gradient (float64) for samples x [n, 8], y [n]."""
    return loss_grad_rounded(x, y, bf16(w))


def loss_grad_rounded(x: np.ndarray, y: np.ndarray, q: np.ndarray):
    """The same for weights already rounded (float64, no further rounding)."""
    w1, b1, w2, b2, w3, b3 = unpack(np.asarray(q, np.float64))
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(y)
    h1 = np.tanh(x @ w1.T + b1)
    h2 = np.tanh(h1 @ w2.T + b2)
    out = h2 @ w3 + b3
    e = out - y
    loss = float(np.mean(e * e))
    dy = 2 * e / n
    d2 = np.outer(dy, w3) * (1 - h2 * h2)
    d1 = (d2 @ w2) * (1 - h1 * h1)
    g = np.zeros(NP)
    g[W1:B1] = (d1.T @ x).reshape(-1)
    g[B1:W2] = d1.sum(0)
    g[W2:B2] = (d2.T @ h1).reshape(-1)
    g[B2:W3] = d2.sum(0)
    g[W3:B3] = dy @ h2
    g[B3] = dy.sum()
    return loss, g


def forward(x: np.ndarray, w: np.ndarray) -> np.ndarray:
    w1, b1, w2, b2, w3, b3 = unpack(bf16(w))
    h1 = np.tanh(np.asarray(x, np.float64) @ w1.T + b1)
    return np.tanh(h1 @ w2.T + b2) @ w3 + b3
