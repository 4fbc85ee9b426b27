"""CPU restatement of the surrogate network's arithmetic (test infrastructure).

Only tests/ import this file: it checks the GPU kernels of
eemd4cuda_b200/csrc/surrogate.cu.  The network has no counterpart in the
reference (which has no learned component); the arithmetic here is the
textbook one: a 1-D convolution with kernel 3, dilation d and zero padding,
channels-last, y[t][n] = b[n] + sum_{tap,c} w[n][tap][c] x[t + (tap-1) d][c],
its input and weight gradients, ReLU, the mean squared error of a residual
prediction, and Adam (Kingma & Ba 2015).
"""
from __future__ import annotations

import numpy as np


def conv(x, w, b=None, dil=1, direction=1):
    """x [B][T][C], w [N][3][C] -> y [B][T][N] (float64)."""
    B, T, C = x.shape
    N = w.shape[0]
    y = np.zeros((B, T, N))
    for tap in range(3):
        s = direction * (tap - 1) * dil
        src = np.zeros_like(x, dtype=np.float64)
        lo, hi = max(0, -s), min(T, T - s)
        if hi > lo:
            src[:, lo:hi] = x[:, lo + s:hi + s]
        y += src @ w[:, tap, :].T
    if b is not None:
        y += b
    return y


def conv_input_grad(dy, w, dil=1):
    """d/dx of conv for upstream dy [B][T][N]: [B][T][C]."""
    wt = np.transpose(w, (2, 1, 0))  # [C][3][N]
    return conv(dy, wt, None, dil, direction=-1)


def conv_weight_grad(dy, x, dil=1):
    """dw [N][3][C], db [N]."""
    B, T, C = x.shape
    N = dy.shape[2]
    dw = np.zeros((N, 3, C))
    for tap in range(3):
        s = (tap - 1) * dil
        src = np.zeros_like(x, dtype=np.float64)
        lo, hi = max(0, -s), min(T, T - s)
        if hi > lo:
            src[:, lo:hi] = x[:, lo + s:hi + s]
        dw[:, tap, :] = np.einsum("btn,btc->nc", dy, src)
    return dw, dy.sum(axis=(0, 1))


def mse_residual(out, base, target, cv, margin):
    """loss and d loss/d out over channels < cv and time [margin, T-margin)."""
    B, T, C = out.shape
    d = base + out - target
    mask = np.zeros_like(d)
    mask[:, margin:T - margin, :cv] = 1.0
    count = B * (T - 2 * margin) * cv
    return float(np.sum((d * mask) ** 2) / count), 2.0 * d * mask / count


def adam(p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
