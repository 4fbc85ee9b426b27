"""The seeded synthetic workloads (CPU): sizes, determinism and the choices
the workload descriptions leave open, as the generators document them."""
import numpy as np

from eemd4cuda_b200 import signals


def test_plain_8k_shape_and_determinism():
    a, b = signals.plain_emd_8k(), signals.plain_emd_8k()
    assert a.shape == (8192,) and a.dtype == np.float64 and np.array_equal(a, b)


def test_harmonic_clicks_levels():
    N = 48000
    x = signals.harmonic_clicks(N, seed=1)
    assert np.array_equal(x, signals.harmonic_clicks(N, seed=1))
    assert not np.array_equal(x, signals.harmonic_clicks(N, seed=2))
    t = np.arange(N) / 48000.0
    tone = sum(np.sin(2 * np.pi * 220.0 * k * t) / k for k in range(1, 9))
    rest = x - tone
    # clicks: 5 onsets, each a jump of the tone's peak
    onsets = np.flatnonzero(np.diff(rest) > 0.5 * np.max(np.abs(tone)))
    assert 1 <= len(onsets) <= 5
    # pink noise 30 dB below the tone RMS (measured away from the clicks' tails)
    quiet = np.ones(N, dtype=bool)
    for o in onsets:
        quiet[o:o + 2000] = False
    ratio = np.sqrt(np.mean(rest[quiet] ** 2)) / np.sqrt(np.mean(tone ** 2))
    assert 10 ** (-32 / 20) < ratio < 10 ** (-28 / 20)


def test_uneven_batch_lengths():
    n = signals.uneven_lengths()
    assert n.shape == (512,) and n.min() >= 4096 and n.max() <= 262144
    assert np.array_equal(n, signals.uneven_lengths())
    assert 25e6 < n.sum() < 40e6  # about 512 x 62k samples


def test_amfm_shape_and_bounds():
    x = signals.amfm_long(1 << 16, seed=2)
    assert x.shape == (1 << 16,) and np.array_equal(x, signals.amfm_long(1 << 16, seed=2))
    assert np.max(np.abs(x)) <= 6 * 1.5  # 6 components of amplitude at most 1 + 0.5
