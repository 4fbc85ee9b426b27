"""The IMF spectra stage on the device, with the reference's interface
(audio_eemd/spectra.py:18-58): stft_block, hilbert_if, if_stats.

stft_block and hilbert_if take one signal (1-D) or a batch of rows (2-D,
[M, N]) as host arrays and return host arrays, like the reference; the
*_device variants take and return float64 torch tensors resident on the GPU,
so the IMFs of eemd_finalize can be analysed without leaving the device.
All arithmetic runs in libeemd_spectra.so (its own Stockham / Bluestein FFT
kernels and the kernels between the transforms; no FFT library); if_stats is
the reference's host reduction.
"""
from __future__ import annotations

import functools
import warnings

import numpy as np

from . import _sp

__all__ = ["stft_block", "hilbert_if", "if_stats", "stft_device", "hilbert_if_device"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the spectra stage needs a CUDA device")
    return torch


@functools.lru_cache(maxsize=64)
def _hilbert_ws(M, N):
    return _sp.hilbert_workspace(M, N)


def hilbert_if_device(x, sr):
    """x: float64 CUDA tensor [M, N] (or [N]) -> (inst_freq, inst_amp) of the same shape."""
    torch = _torch()
    x2 = x.reshape(1, -1) if x.dim() == 1 else x
    x2 = x2.contiguous()
    M, N = int(x2.shape[0]), int(x2.shape[1])
    if N < 2:
        raise ValueError("hilbert_if needs at least 2 samples")
    freq = torch.empty_like(x2)
    amp = torch.empty_like(x2)
    ws = torch.empty((_hilbert_ws(M, N),), dtype=torch.uint8, device=x2.device)
    _sp.hilbert_if(x2, M, N, sr, freq, amp, ws)
    return freq.reshape(x.shape), amp.reshape(x.shape)


# arrays up to this size move through pinned tensors of the call (torch's
# caching host allocator keeps their blocks for reuse); larger ones through
# pageable memory, so that large calls leave no large pinned blocks behind
PINNED_BYTES = 64 << 20


def _to_device(torch, a):
    """A host array on the device: through a pinned copy (asynchronous
    upload) up to PINNED_BYTES, else a pageable copy."""
    if a.nbytes > PINNED_BYTES:
        return torch.from_numpy(a).to("cuda")
    h = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    h.numpy()[...] = a
    return h.to("cuda", non_blocking=True)


def _to_host(torch, *ts):
    """Device tensors as host arrays: views of pinned tensors of this call
    (torch's caching host allocator) with one synchronisation, or pageable
    copies for tensors above PINNED_BYTES."""
    hs = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
          if t.numel() * t.element_size() <= PINNED_BYTES else None for t in ts]
    for h, t in zip(hs, ts):
        if h is not None:
            h.copy_(t, non_blocking=True)
    out = [t.cpu() if h is None else None for h, t in zip(hs, ts)]  # (each synchronises)
    torch.cuda.current_stream().synchronize()
    return tuple((h if h is not None else o).numpy() for h, o in zip(hs, out))


def hilbert_if(imf, sr):
    """Instantaneous frequency [Hz] and amplitude of one IMF (or of each row):
    z = imf + i H(imf), d/dt arg(z) / 2 pi, |z| (spectra.py:32-45)."""
    torch = _torch()
    a = np.ascontiguousarray(imf, dtype=np.float64)
    f, A = hilbert_if_device(_to_device(torch, a), sr)
    return _to_host(torch, f, A)


def _segments(N, nperseg, noverlap):
    # the default overlap is half the requested frame (spectra.py:25-26),
    # filled in before scipy's rule cuts a frame longer than the input to the
    # input (with a warning); a short input with the default overlap is
    # therefore an error, as in the reference
    if noverlap is None:
        noverlap = nperseg // 2
    if nperseg > N:
        warnings.warn(f"nperseg = {nperseg} is greater than input length  = {N}, using nperseg = {N}")
        nperseg = N
    if noverlap >= nperseg:
        raise ValueError("noverlap must be less than nperseg.")
    return int(nperseg), int(noverlap)


@functools.lru_cache(maxsize=64)
def _stft_plan(M, N, nperseg, noverlap):
    """(F, T, workspace bytes) of one STFT shape (queried once per shape)."""
    F, T = _sp.stft_shape(N, nperseg, noverlap)
    return F, T, _sp.stft_workspace(M, N, nperseg, noverlap)


@functools.lru_cache(maxsize=64)
def _stft_axes(nperseg, noverlap, T, sr):
    f = np.fft.rfftfreq(nperseg, 1.0 / sr)
    t = np.arange(T) * (nperseg - noverlap) / float(sr)
    f.flags.writeable = False
    t.flags.writeable = False
    return f, t


def stft_device(x, sr, nperseg=4096, noverlap=None):
    """x: float64 CUDA tensor [M, N] (or [N]) -> (f, t, Z complex128 [M, F, T] (or [F, T]))."""
    torch = _torch()
    x2 = (x.reshape(1, -1) if x.dim() == 1 else x).contiguous()
    M, N = int(x2.shape[0]), int(x2.shape[1])
    nperseg, noverlap = _segments(N, nperseg, noverlap)
    F, T, wsb = _stft_plan(M, N, nperseg, noverlap)
    Z = torch.empty((M, F, T), dtype=torch.complex128, device=x2.device)
    ws = torch.empty((wsb,), dtype=torch.uint8, device=x2.device)
    _sp.stft(x2, M, N, nperseg, noverlap, Z, ws)
    f, t = _stft_axes(nperseg, noverlap, T, float(sr))
    return f.copy(), t.copy(), (Z[0] if x.dim() == 1 else Z)


def stft_block(x, sr, nperseg=4096, noverlap=None):
    """STFT of a signal (or of each row): Hann window, 50 % overlap by
    default, zero-extended ends, one-sided (spectra.py:18-29).  Returns (f, t, Zxx)."""
    torch = _torch()
    a = np.ascontiguousarray(x, dtype=np.float64)
    f, t, Z = stft_device(_to_device(torch, a), sr, nperseg, noverlap)
    return f, t, _to_host(torch, Z)[0]


def if_stats(w: np.ndarray) -> dict:
    """Median / IQR of an IF series, positive part only (spectra.py:48-58)."""
    wp = w[w > 0]
    if wp.size == 0:
        return {"median": None, "iqr": None, "n_pos_frac": 0.0}
    lo, hi = np.percentile(wp, [25, 75])
    return {"median": float(np.median(wp)), "iqr": float(hi - lo), "n_pos_frac": float(wp.size / w.size)}
