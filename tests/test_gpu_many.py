"""decompose_many: many signals of uneven length in one launch per trial
batch, against decompose of each signal alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
pytest.importorskip("torch")

from eemd4cuda_b200 import emd_par as M  # noqa: E402
from eemd4cuda_b200 import signals  # noqa: E402


def batch():
    return [signals.harmonic_clicks(n, seed=100 + i, fs=8000.0) for i, n in enumerate([3000, 8192, 1500, 5000])]


def test_emd_of_many_equals_emd_of_each():
    xs = batch()
    many = M.decompose_many(xs, E=1, tau=0.25, max_sifts=50, max_imf=10, exact=True)
    for x, r in zip(xs, many):
        one = M.decompose(x, E=1, tau=0.25, max_sifts=50, max_imf=10, exact=True)
        assert r.n_modes == one.n_modes
        assert np.array_equal(r.imfs, one.imfs)
        assert np.max(np.abs(r.residual - one.residual)) <= 1e-12 * np.abs(x).max()
        assert r.stats["per_trial_total_sifts"].tolist() == one.stats["per_trial_total_sifts"].tolist()


def test_eemd_of_many():
    xs = batch()
    many = M.decompose_many(xs, E=8, seed=3, tau=0.25, max_sifts=20, max_imf=8, dtype=np.float32)
    for x, r in zip(xs, many):
        assert r.imfs.shape == (r.n_modes, len(x))
        x32 = x.astype(np.float32).astype(np.float64)  # the engine decomposed the float32 signal
        assert np.max(np.abs(x32 - r.imfs.sum(axis=0) - r.residual)) <= 1e-12 * np.abs(x).max()
        assert len(r.stats["per_trial_total_sifts"]) == 8
    # signal 0's noise stream is the one decompose draws for a lone signal
    one = M.decompose(xs[0], E=8, seed=3, tau=0.25, max_sifts=20, max_imf=8, dtype=np.float32)
    assert one.n_modes == many[0].n_modes and np.array_equal(one.imfs, many[0].imfs)
    # trial batches: two launches of 4 trials add up to the same sums
    half = M.decompose_many(xs, E=8, seed=3, tau=0.25, max_sifts=20, max_imf=8, dtype=np.float32, batch=4)
    for a, b in zip(many, half):
        assert a.n_modes == b.n_modes and np.array_equal(a.imfs, b.imfs)
