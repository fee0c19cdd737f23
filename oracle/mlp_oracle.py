"""TEST INFRASTRUCTURE ONLY -- the checker of the learned planner's network.

A float64 numpy restatement of the MLP that partitioned_join_b200's
pj_mlp_forward / pj_mlp_backward / pj_mlp_mse_grad / pj_mlp_adam kernels
compute (csrc/pj_learn.cu): in -> h1 (ReLU) -> h2 (ReLU) -> out, parameters
in one vector W1[in][h1], b1, W2[h1][h2], b2, W3[h2][out], b3.  Gradients by
the chain rule; Adam as Kingma and Ba (2015) with bias correction.  The
reference has no learned planner; this file pins the library's own kernels.
"""
from __future__ import annotations

import numpy as np


def split(params: np.ndarray, d_in: int, h1: int, h2: int, out: int):
    p = np.asarray(params, dtype=np.float64)
    sizes = [d_in * h1, h1, h1 * h2, h2, h2 * out, out]
    parts, o = [], 0
    for s in sizes:
        parts.append(p[o:o + s])
        o += s
    assert o == p.shape[0]
    W1, b1, W2, b2, W3, b3 = parts
    return W1.reshape(d_in, h1), b1, W2.reshape(h1, h2), b2, W3.reshape(h2, out), b3


def param_count(d_in, h1, h2, out):
    return d_in * h1 + h1 + h1 * h2 + h2 + h2 * out + out


def forward(params, x, d_in, h1, h2, out):
    W1, b1, W2, b2, W3, b3 = split(params, d_in, h1, h2, out)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1 + b1
    a1 = np.maximum(z1, 0)
    z2 = a1 @ W2 + b2
    a2 = np.maximum(z2, 0)
    y = a2 @ W3 + b3
    return y, (x, z1, a1, z2, a2)


def backward(params, cache, dy, d_in, h1, h2, out):
    W1, b1, W2, b2, W3, b3 = split(params, d_in, h1, h2, out)
    x, z1, a1, z2, a2 = cache
    dy = np.asarray(dy, dtype=np.float64)
    dW3 = a2.T @ dy
    db3 = dy.sum(0)
    da2 = dy @ W3.T
    dz2 = da2 * (z2 > 0)
    dW2 = a1.T @ dz2
    db2 = dz2.sum(0)
    da1 = dz2 @ W2.T
    dz1 = da1 * (z1 > 0)
    dW1 = x.T @ dz1
    db1 = dz1.sum(0)
    return np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])


def mse_grad(y, target, mask=None):
    y = np.asarray(y, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    m = np.ones_like(y) if mask is None else np.asarray(mask, dtype=np.float64)
    denom = max(m.sum(), 1.0)
    d = y - t
    return 2 * d * m / denom, float((m * d * d).sum() / denom)


def adam(p, g, m, v, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
