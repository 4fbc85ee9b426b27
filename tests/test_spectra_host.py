"""Host-side rules of the spectra stage (no GPU): the frame/overlap rules of
stft_block (audio_eemd/spectra.py:18-29 over scipy.signal.stft), and the
oracle's restatement against scipy itself at the frame lengths, hops and
signal lengths the GPU edge tests use."""
import warnings

import numpy as np
import pytest

from oracle import spectra_oracle as SP

pytest.importorskip("torch")
from eemd4cuda_b200 import spectra  # noqa: E402


def test_frame_and_overlap_rules():
    # default: half the frame
    assert spectra._segments(48000, 4096, None) == (4096, 2048)
    assert spectra._segments(5000, 1000, 333) == (1000, 333)
    # a frame longer than the signal is cut to it, with scipy's warning
    with pytest.warns(UserWarning, match="greater than input length"):
        assert spectra._segments(1000, 4096, 300) == (1000, 300)
    # ... and the default overlap, half the requested frame, is then too long
    with pytest.warns(UserWarning), pytest.raises(ValueError, match="noverlap must be less than nperseg"):
        spectra._segments(1000, 4096, None)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        with pytest.raises(ValueError, match="noverlap"):
            spectra._segments(5000, 1000, 1000)


@pytest.mark.parametrize("N,nper,nov", [(3000, 256, None), (4097, 512, 384), (5000, 1000, 333),
                                        (4096, 512, 384), (777, 64, 1), (20000, 4096, 0), (1000, 1000, 300)])
def test_oracle_stft_equals_scipy(N, nper, nov):
    """The reference's call: Hann window, boundary='zeros', padded=False."""
    ss = pytest.importorskip("scipy.signal")
    x = np.random.default_rng(N).standard_normal(N)
    sr = 48000
    f, t, Z = SP.stft(x, sr, nper, nov)
    rf, rt, rZ = ss.stft(x, fs=sr, window="hann", nperseg=nper, noverlap=nper // 2 if nov is None else nov,
                         boundary="zeros", padded=False)
    assert Z.shape == rZ.shape
    assert np.allclose(f, rf, rtol=0, atol=1e-9) and np.allclose(t, rt, rtol=0, atol=1e-12)
    assert np.max(np.abs(Z - rZ)) <= 1e-12 * np.max(np.abs(rZ))


@pytest.mark.parametrize("N", [2, 3, 5, 8, 31, 33, 1001, 4097])
def test_oracle_hilbert_equals_scipy(N):
    """The analytic signal of even and odd lengths, and the reference's IF
    formula on it (unwrap of the angle, np.gradient, / 2 pi)."""
    ss = pytest.importorskip("scipy.signal")
    x = np.random.default_rng(N).standard_normal(N)
    sr = 48000
    w, A = SP.hilbert_if(x, sr)
    z = ss.hilbert(x)
    assert np.max(np.abs(A - np.abs(z))) <= 1e-12 * max(1.0, np.abs(z).max())
    rw = np.gradient(np.unwrap(np.angle(z)), 1.0 / sr) / (2.0 * np.pi)
    assert np.max(np.abs(w - rw)) <= 1e-6 * sr
