"""CPU restatement of the IMF spectra stage -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/ (and bench.py's CPU-baseline leg): it checks the GPU
kernels of eemd4cuda_b200/csrc/spectra.cu.  The reference computes these in
audio_eemd/spectra.py with scipy.signal (no version pinned in the reference;
this container has scipy 1.x with pocketfft):

  spectra.py:18-29  stft_block -> scipy.signal.stft(window='hann',
                    boundary='zeros', padded=False)              -> stft()
  spectra.py:32-45  hilbert_if -> scipy.signal.hilbert, np.unwrap(np.angle),
                    np.gradient(phase, 1/sr) / 2pi, |z|          -> hilbert_if()
  spectra.py:48-58  if_stats                                     -> if_stats()

Restated from the published algorithms with numpy: the analytic signal is
ifft(fft(x) * h), h = 1 at DC (and Nyquist for even N), 2 on the positive
frequencies, 0 on the negative ones (scipy.signal.hilbert); the STFT frames
the signal extended by nperseg//2 zeros at both ends with hop
nperseg - noverlap, multiplies by the periodic Hann window
0.5 - 0.5 cos(2 pi n / nperseg), takes the one-sided FFT and divides by the
window's sum (scipy's 'spectrum' scaling for mode 'stft').  Pinned against
fixtures made by the reference's own functions
(tests/golden/make_spectra_golden.py).
"""
from __future__ import annotations

import numpy as np


def analytic(x):
    x = np.asarray(x, dtype=float)
    N = x.shape[-1]
    h = np.zeros(N)
    if N % 2 == 0:
        h[0] = h[N // 2] = 1.0
        h[1:N // 2] = 2.0
    else:
        h[0] = 1.0
        h[1:(N + 1) // 2] = 2.0
    return np.fft.ifft(np.fft.fft(x, axis=-1) * h, axis=-1)


def hilbert_if(imf, sr):
    z = analytic(imf)
    phase = np.unwrap(np.angle(z))
    return np.gradient(phase, 1.0 / sr) / (2.0 * np.pi), np.abs(z)


def hann_periodic(n):
    return 0.5 - 0.5 * np.cos(2.0 * np.pi * np.arange(n) / n)


def stft(x, sr, nperseg=4096, noverlap=None):
    """(f, t, Z [F, T]) of one signal."""
    if noverlap is None:
        noverlap = nperseg // 2
    x = np.asarray(x, dtype=float)
    w = hann_periodic(nperseg)
    half = nperseg // 2
    ext = np.concatenate([np.zeros(half), x, np.zeros(half)])
    step = nperseg - noverlap
    T = (len(ext) - noverlap) // step
    frames = np.stack([ext[j * step:j * step + nperseg] * w for j in range(T)])
    Z = np.fft.rfft(frames, axis=-1) / w.sum()
    f = np.fft.rfftfreq(nperseg, 1.0 / sr)
    t = np.arange(T) * step / float(sr)
    return f, t, Z.T


def if_stats(w):
    wp = w[w > 0]
    if wp.size == 0:
        return {"median": None, "iqr": None, "n_pos_frac": 0.0}
    lo, hi = np.percentile(wp, [25, 75])
    return {"median": float(np.median(wp)), "iqr": float(hi - lo), "n_pos_frac": float(wp.size / w.size)}
