"""Oracle (test infrastructure): the warm-start MLP in FP64 NumPy -- forward, loss, backward, AdamW.

The network is the learned part of the LM warm start (no reference counterpart; its specification
is a 1024 -> 256 -> 256 -> 7 MLP with ReLU, trained by AdamW on a weighted mean-squared error).
The GPU implementation computes the same quantities with bf16 operands and f32 accumulation; tests
feed this oracle the same bf16-rounded inputs and weights and compare within bf16 tolerances.
"""

from __future__ import annotations

import numpy as np


def forward(x, w1, b1, w2, b2, w3, b3):
    """x (B, 1024) -> (h1, h2, y)."""
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    y = h2 @ w3.T + b3
    return h1, h2, y


def loss_and_grad_output(y, t, weights):
    """L = mean over the batch of sum_j w_j (y_j - t_j)^2, and dL/dy."""
    d = y - t
    loss = float(np.mean(np.sum(weights * d * d, axis=1)))
    return loss, 2.0 * weights * d / y.shape[0]


def backward(x, h1, h2, dy, w2, w3):
    """Gradients of the loss (given dL/dy) with respect to w1, b1, w2, b2, w3, b3."""
    gw3 = dy.T @ h2
    gb3 = dy.sum(axis=0)
    dh2 = (dy @ w3) * (h2 > 0)
    gw2 = dh2.T @ h1
    gb2 = dh2.sum(axis=0)
    dh1 = (dh2 @ w2) * (h1 > 0)
    gw1 = dh1.T @ x
    gb1 = dh1.sum(axis=0)
    return gw1, gb1, gw2, gb2, gw3, gb3


def adamw(w, g, m, v, step, *, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
    """One decoupled-weight-decay Adam step (Loshchilov & Hutter); returns (w, m, v)."""
    m = beta1 * m + (1.0 - beta1) * g
    v = beta2 * v + (1.0 - beta2) * g * g
    mh = m / (1.0 - beta1 ** step)
    vh = v / (1.0 - beta2 ** step)
    w = w - lr * (mh / (np.sqrt(vh) + eps) + weight_decay * w)
    return w, m, v


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isnan(a), np.nan, out)
