"""CPU restatement of the surrogate network's arithmetic (test infrastructure).

Only tests/ import this file: it checks the GPU kernels of
eemd4cuda_b200/csrc/surrogate.cu.  The network has no counterpart in the
reference (which has no learned component); the arithmetic here is the
textbook one: a 1-D convolution with kernel 3, dilation d and zero padding,
channels-last, y[t][n] = b[n] + sum_{tap,c} w[n][tap][c] x[t + (tap-1) d][c],
its input and weight gradients, ReLU, the mean squared error of a residual
prediction, and Adam (Kingma & Ba 2015); and the surrogate's input and
output stages: per-mode ensemble means and the residual x - sum(means) (the
order of emd_par.py:241-250 in the reference), scaled by the signal's RMS,
and the served decomposition with its reconstruction error and Huang et al.
(1998) orthogonality index.
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


def project_outputs(w, b=None):
    """Weights w[N][3][C] (and bias b[N]) minus their mean over N: the layer's
    outputs then sum to zero over its output channels."""
    w = w - w.mean(axis=0, keepdims=True)
    return w if b is None else (w, b - b.mean())


def mse_residual(out, base, target, cv, margin, project=False, delta=0.0, weights=None):
    """loss and d loss/d out over channels < cv and time [margin, T-margin):
    the mean of d^2 (d = base + out - target), or with delta > 0 of the Huber
    loss (d^2 within delta, 2 delta |d| - delta^2 beyond), each channel times
    weights[c]; project removes each sample's mean over the cv channels from
    the gradient."""
    B, T, C = out.shape
    d = (0.0 if base is None else base) + out - target
    mask = np.zeros_like(d)
    mask[:, margin:T - margin, :cv] = 1.0 if weights is None else np.asarray(weights, np.float64)[:cv]
    count = B * (T - 2 * margin) * cv
    if delta > 0:
        big = np.abs(d) > delta
        el = np.where(big, 2 * delta * np.abs(d) - delta * delta, d * d)
        g = 2.0 * np.where(big, np.sign(d) * delta, d) * mask / count
    else:
        el = d * d
        g = 2.0 * d * mask / count
    if project:
        g[..., :cv] -= g[..., :cv].mean(axis=-1, keepdims=True)
    return float(np.sum(el * mask) / count), g


def adam(p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8, max_norm=0.0):
    """Adam; max_norm > 0 first scales g to that Euclidean norm at most (a
    non-finite norm skips the step)."""
    if max_norm > 0:
        nrm = float(np.sqrt(np.sum(np.asarray(g, np.float64) ** 2)))
        if not np.isfinite(nrm):
            return p, m, v
        if nrm > max_norm:
            g = g * (max_norm / nrm)
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v


def rms(x):
    """[S][N] -> [S] (1 for a zero signal)."""
    r = np.sqrt(np.mean(np.asarray(x, np.float64) ** 2, axis=1))
    return np.where(r > 0, r, 1.0)


def means_and_residual(imf_sum, count, x):
    """imf_sum [S][K][N], count [S][K], x [S][N] -> means [S][K][N], resid [S][N]
    (the residual summed in mode order)."""
    means = imf_sum / np.maximum(count, 1)[:, :, None]
    acc = np.zeros_like(means[:, 0])
    for m in range(means.shape[1]):
        acc = acc + means[:, m]
    return means, np.asarray(x, np.float64) - acc


def prepare(imf_sum, count, x, scale, C=16):
    """Network input [S][N][C] (float64, before the bf16 rounding)."""
    means, resid = means_and_residual(imf_sum, count, x)
    S, K, N = means.shape
    out = np.zeros((S, N, C))
    out[:, :, :K] = np.transpose(means, (0, 2, 1)) / scale[:, None, None]
    out[:, :, K] = resid / scale[:, None]
    return out


def orthogonality_index(components, x):
    """Huang et al. (1998): sum over pairs j != k of <c_j, c_k> / ||x||^2."""
    g = components @ components.T
    return float((g.sum() - np.trace(g)) / max(float(x @ x), 1e-300))


def combine(imf_sum, count, x, scale, net, P):
    """Served IMFs [S][K][N] and residual [S][N] from the network output
    net [S][N][C] (corrections of the first P modes, their sum taken from the
    residual), with per-signal reconstruction error and orthogonality indices
    of the P corrected modes, of all IMFs and the residual, and of the first P
    small-ensemble means."""
    means, resid = means_and_residual(imf_sum, count, x)
    S, K, N = means.shape
    d = np.zeros((S, K, N))
    d[:, :P] = scale[:, None, None] * np.transpose(net[:, :, :P], (0, 2, 1))
    imfs = means + d
    moved = np.zeros((S, N))
    for m in range(K):
        moved = moved + d[:, m]
    res = resid - moved
    x = np.asarray(x, np.float64)
    recon = np.array([np.linalg.norm(x[s] - imfs[s].sum(axis=0) - res[s]) / np.linalg.norm(x[s])
                      for s in range(S)])
    io_p = np.array([orthogonality_index(imfs[s][:P], x[s]) for s in range(S)])
    io = np.array([orthogonality_index(np.vstack([imfs[s], res[s][None]]), x[s]) for s in range(S)])
    io_ref = np.array([orthogonality_index(means[s][:P], x[s]) for s in range(S)])
    return imfs, res, recon, io_p, io, io_ref
