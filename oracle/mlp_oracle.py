"""CPU oracle of the warm-start MLP (forward, loss, backward).

TEST INFRASTRUCTURE ONLY: checks the project's BF16 GPU training kernels.
Network: x (128 padded inputs) -> h0 = relu(W0 x + b0) -> 3 residual blocks
h_l = h_{l-1} + relu(W_l h_{l-1} + b_l) -> y = W4 h3 + b4 (+ IDW base).
Loss: shock-weighted relative MSE of loss.py:20-23 with fixed per-variable
denominators. ``bf16=True`` rounds every tensor the GPU stores in BF16 at the
same points (weights, inputs, z, h, dh, dz); arithmetic is float64.
"""
from __future__ import annotations

import numpy as np


def bf16_round(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32).copy()
    u = f.view(np.uint32)
    u += np.uint32(0x7FFF) + ((u >> np.uint32(16)) & np.uint32(1))
    u &= np.uint32(0xFFFF0000)
    return f.astype(np.float64)


def forward(params, X, base=None, bf16=True):
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    W0, b0 = params['W0'], params['b0']
    x = r(X)
    z = [None] * 4
    h = [None] * 4
    z[0] = x @ r(W0).T + b0
    h[0] = r(np.maximum(z[0], 0.0))
    z[0] = r(z[0])
    for l in range(1, 4):
        zl = h[l - 1] @ r(params[f'W{l}']).T + params[f'b{l}']
        h[l] = r(h[l - 1] + np.maximum(zl, 0.0))
        z[l] = r(zl)
    y = h[3] @ params['W4'].T + params['b4']
    if base is not None:
        y = y + base
    return y, dict(x=x, z=z, h=h)


def loss_and_grad(y, tgt, w, inv_den):
    R = y.shape[0]
    d = y - tgt
    wr = np.ones(R) if w is None else w
    L = float(np.sum(wr[:, None] * d * d * inv_den[None, :]) / (4 * R))
    dy = 2.0 * wr[:, None] * d * inv_den[None, :] / (4 * R)
    return L, dy


def backward(params, acts, dy, bf16=True):
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    g = {}
    h, z, x = acts['h'], acts['z'], acts['x']
    g['W4'] = dy.T @ h[3]
    g['b4'] = dy.sum(0)
    dh_f = dy @ params['W4']
    dh = r(dh_f)
    dz = r(dh_f * (z[3] > 0))
    for l in (3, 2, 1):
        g[f'W{l}'] = dz.T @ h[l - 1]
        g[f'b{l}'] = dz.sum(0)
        acc = dz @ r(params[f'W{l}']) + dh
        dh = r(acc)
        dz = r(acc * (z[l - 1] > 0))
    g['W0'] = dz.T @ x
    g['b0'] = dz.sum(0)
    return g
