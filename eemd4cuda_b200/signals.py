"""Seeded synthetic signals with the shapes of the benchmark workloads.

No public dataset is named for these workloads; each generator below fixes
the choices the workload description leaves open (pink-noise level, click
shape, AM/FM rates) so that every run sees the same input bits.

  plain_emd_8k()        N=8192 @ 8 kHz: 50 Hz + 400 Hz tones, 1->2 kHz linear
                        chirp (amplitude 0.3), Gaussian noise sigma 0.01, seed 0
  harmonic_clicks(N)    f0=220 Hz tone with 8 partials of amplitude 1/k, pink
                        noise 30 dB below the tone RMS, 5 exponentially decaying
                        clicks (tau 2 ms, amplitude = tone peak) @ 48 kHz
  amfm_long(N)          6 AM/FM components, carriers log-uniform 10 Hz-20 kHz,
                        AM depth U(0,0.5), FM index U(0,2), modulation rates
                        log-uniform 0.1-20 Hz, unit amplitudes @ 48 kHz
  uneven_batch()        512 lengths log-uniform in [4096, 262144] (seed 4),
                        signal i = harmonic_clicks(N_i, seed=1000+i)
"""
from __future__ import annotations

import numpy as np


def plain_emd_8k(N: int = 8192, fs: float = 8000.0, seed: int = 0) -> np.ndarray:
    t = np.arange(N) / fs
    T = N / fs
    x = (0.8 * np.sin(2 * np.pi * 50 * t) + 0.5 * np.sin(2 * np.pi * 400 * t + 0.3)
         + 0.3 * np.sin(2 * np.pi * (1000 * t + 500 * t * t / T)))
    return x + 0.01 * np.random.default_rng(seed).standard_normal(N)


def _pink(rng: np.random.Generator, N: int) -> np.ndarray:
    """Gaussian noise with a 1/f power spectrum (unit RMS)."""
    w = rng.standard_normal(N)
    W = np.fft.rfft(w)
    f = np.arange(W.shape[0], dtype=float)
    f[0] = 1.0
    W = W / np.sqrt(f)
    W[0] = 0.0
    p = np.fft.irfft(W, n=N)
    return p / np.sqrt(np.mean(p * p))


def harmonic_clicks(N: int = 48000, seed: int = 1, fs: float = 48000.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(N) / fs
    tone = np.zeros(N)
    for k in range(1, 9):
        tone += np.sin(2 * np.pi * 220.0 * k * t) / k
    rms = np.sqrt(np.mean(tone * tone))
    peak = np.max(np.abs(tone))
    x = tone + _pink(rng, N) * rms * 10 ** (-30 / 20)
    tau = 0.002 * fs
    n = np.arange(N)
    for n0 in rng.integers(0, N, size=5):
        m = n >= n0
        x[m] += peak * np.exp(-(n[m] - n0) / tau)
    return x


def amfm_long(N: int = 1 << 22, seed: int = 2, fs: float = 48000.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(N) / fs
    x = np.zeros(N)
    for _ in range(6):
        fc = np.exp(rng.uniform(np.log(10.0), np.log(20000.0)))
        a = rng.uniform(0.0, 0.5)
        beta = rng.uniform(0.0, 2.0)
        fa = np.exp(rng.uniform(np.log(0.1), np.log(20.0)))
        fm = np.exp(rng.uniform(np.log(0.1), np.log(20.0)))
        pa, pm, ph = rng.uniform(0.0, 2 * np.pi, size=3)
        x += (1.0 + a * np.sin(2 * np.pi * fa * t + pa)) * \
            np.sin(2 * np.pi * fc * t + beta * np.sin(2 * np.pi * fm * t + pm) + ph)
    return x


def uneven_lengths(count: int = 512, lo: int = 4096, hi: int = 262144, seed: int = 4) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)


def uneven_batch(count: int = 512, seed: int = 4):
    lengths = uneven_lengths(count, seed=seed)
    return [harmonic_clicks(int(n), seed=1000 + i) for i, n in enumerate(lengths)]


def two_tones(sr: int = 8000, seconds: float = 4.0):
    """100 Hz + 105 Hz mode-mixing pair (audio_eemd/tests/conftest.py:41-46)."""
    t = np.arange(int(seconds * sr)) / sr
    return (np.sin(2 * np.pi * 100 * t) + np.sin(2 * np.pi * 105 * t)) / 2, sr


def modulated_chirp(N: int = 441000, fs: float = 44100.0):
    """Strongly modulated chirp with pathological knot spacing
    (test_phase3_gates.py:200-206: f(t) = 50(1 + 0.95 sin(2 pi t / 8 s)))."""
    t = np.arange(N) / fs
    f = 50.0 * (1.0 + 0.95 * np.sin(2 * np.pi * t / 8.0))
    phi = 2 * np.pi * np.cumsum(f) / fs
    return np.sin(phi) + 0.01 * np.random.default_rng(0).standard_normal(N)
