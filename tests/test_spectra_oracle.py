"""The spectra restatement (oracle/spectra_oracle.py) against fixtures made by
the reference's own audio_eemd/spectra.py (tests/golden/make_spectra_golden.py)."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import spectra_oracle as SP


@pytest.fixture(scope="module")
def golden():
    d = np.load(GOLDEN / "spectra_cases.npz")
    return {k: d[k] for k in d.files}


def steady(amp, frac=1e-3):
    """samples whose analytic-signal magnitude (and its neighbours') is not
    near zero: elsewhere the phase, hence the frequency, is ill-conditioned"""
    ok = amp > frac * amp.max()
    return ok & np.roll(ok, 1) & np.roll(ok, -1)


@pytest.mark.parametrize("name", ["a", "b", "c"])
def test_oracle_spectra_match_reference(golden, name):
    N, sr, nper, nov = golden[f"{name}_params"].tolist()
    nov = None if nov < 0 else nov
    X = golden[f"{name}_x"]
    for r in range(X.shape[0]):
        f, t, Z = SP.stft(X[r], sr, nper, nov)
        assert np.allclose(f, golden[f"{name}_f"], rtol=0, atol=1e-9)
        assert np.allclose(t, golden[f"{name}_t"], rtol=0, atol=1e-12)
        Zr = golden[f"{name}_{r}_Z"]
        assert Z.shape == Zr.shape
        assert np.max(np.abs(Z - Zr)) <= 1e-12 * np.max(np.abs(Zr))
        w, A = SP.hilbert_if(X[r], sr)
        Ar, wr = golden[f"{name}_{r}_amp"], golden[f"{name}_{r}_if"]
        assert np.max(np.abs(A - Ar)) <= 1e-12 * np.max(Ar)
        m = steady(Ar)
        assert np.max(np.abs(w - wr)[m]) <= 1e-6 * sr
        st = SP.if_stats(w)
        ref = golden[f"{name}_{r}_ifstats"]
        assert abs(st["n_pos_frac"] - ref[2]) <= 2.0 / N
        assert abs(st["median"] - ref[0]) <= 1e-6 * sr
