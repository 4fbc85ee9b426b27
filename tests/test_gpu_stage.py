"""The reference's own stage adapter (audio_eemd/eemd_stage.py, unchanged,
from the reference installed in baseline/_ref) running on this engine
through eemd4cuda_b200/compat/emd_par.py: the reference's five stage tests
(audio_eemd/tests/test_eemd_stage.py:8-69) with method='gpu' where they use
'cpu' (the engine has no CPU method), plus 'auto', and the two-tone
mode-mixing check with this package's Hilbert frequency in place of
audio_eemd.spectra (scipy)."""
import sys

import numpy as np
import pytest

import ref_stage

pytestmark = pytest.mark.gpu
pytest.importorskip("torch")

from eemd4cuda_b200 import signals, spectra  # noqa: E402


@pytest.fixture
def stage(monkeypatch):
    return ref_stage.load(monkeypatch)


@pytest.fixture(scope="module")
def two_tones():
    return signals.two_tones()


def dominant_freq(x, sr):
    """periodogram peak (DC excluded), as the reference's report computes it"""
    X = np.abs(np.fft.rfft(x * np.hanning(len(x))))
    f = np.fft.rfftfreq(len(x), 1.0 / sr)
    return float(f[np.argmax(X[1:]) + 1])


@pytest.mark.parametrize("method", ["gpu", "auto"])
def test_emd_single(stage, two_tones, method):
    x, sr = two_tones
    d = stage.run_eemd(x, method=method, E=1, seed=0)
    # the stage imported this engine's compat module, not the reference's emd_par
    assert sys.modules["emd_par"].__file__ == str(ref_stage.COMPAT / "emd_par.py")
    assert d.n_modes >= 1
    assert d.imfs.shape == (d.n_modes, len(x))
    assert d.residual.shape == (len(x),)
    assert d.recon < 1e-6 * np.abs(x).max()
    assert d.stats["method"] == "gpu" and d.stats["E"] == 1


def test_eemd_ensemble(stage, two_tones):
    x, sr = two_tones
    d = stage.run_eemd(x, method="gpu", E=8, seed=1)
    assert d.n_modes >= 1
    assert d.imfs.shape[0] == d.n_modes and d.imfs.shape[1] == len(x)
    assert d.recon < 1e-6 * np.abs(x).max()
    assert "per_trial_total_sifts" in d.stats
    assert len(d.stats["per_trial_total_sifts"]) == 8


def test_seed_determinism(stage, two_tones):
    x, sr = two_tones
    a = stage.run_eemd(x, method="gpu", E=4, seed=42)
    b = stage.run_eemd(x, method="gpu", E=4, seed=42)
    assert a.n_modes == b.n_modes
    assert np.array_equal(a.imfs, b.imfs) and np.array_equal(a.residual, b.residual)


def test_two_tone_mode_mixing(stage, two_tones):
    """100 / 105 Hz: the carrier stays in one in-band IMF whose Hilbert
    frequency stays in band, and out-of-band IMFs plus residual carry at most
    15 % of the energy (the reference's own bounds)."""
    x, sr = two_tones
    d = stage.run_eemd(x, method="gpu", E=8, seed=1)
    assert d.n_modes >= 2
    dom = [dominant_freq(imf, sr) for imf in d.imfs]
    in_band = np.array([95.0 <= f <= 110.0 for f in dom])
    e = np.sum(d.imfs ** 2, axis=1) / np.sum(x ** 2)
    assert e[in_band].max() >= 0.8, e
    i = int(np.argmax(np.where(in_band, e, 0.0)))
    if0, _ = spectra.hilbert_if(d.imfs[i], sr)
    assert 95.0 <= float(np.median(if0)) <= 110.0
    e_res = float(np.sum(d.residual ** 2) / np.sum(x ** 2))
    assert e[~in_band].sum() + e_res <= 0.15, (e[~in_band].sum(), e_res)


def test_bad_input_raises(stage):
    with pytest.raises(stage.EEMDError) as ei:
        stage.run_eemd(np.ones(5), method="gpu", E=1)
    assert ei.value.code == "eemd.bad_input"


def test_injected_allocation_failure_is_a_backend_error(stage, two_tones, monkeypatch):
    """A device allocation that fails (injected on the host: torch.zeros on the
    device raises the out-of-memory error) surfaces from the reference's stage
    as eemd.backend, and the next call runs normally."""
    import torch
    x, sr = two_tones
    real = torch.zeros

    def failing(*a, **k):
        dev = k.get("device")
        if dev is not None and torch.device(dev).type == "cuda":
            raise torch.OutOfMemoryError("injected allocation failure")
        return real(*a, **k)

    monkeypatch.setattr(torch, "zeros", failing)
    with pytest.raises(stage.EEMDError) as ei:
        stage.run_eemd(x, method="gpu", E=4, seed=1)
    assert ei.value.code == "eemd.backend"
    monkeypatch.setattr(torch, "zeros", real)
    d = stage.run_eemd(x, method="gpu", E=4, seed=1)
    assert d.n_modes >= 1 and d.recon < 1e-6 * np.abs(x).max()
