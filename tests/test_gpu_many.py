"""decompose_many: many signals of uneven length in one launch per trial
batch, against decompose of each signal alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
pytest.importorskip("torch")

from eemd4cuda_b200 import _lib as L  # noqa: E402
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


def test_uneven_batch_against_oracle_per_trial():
    """Eight signals of mixed lengths (4096 - 65536 samples, the uneven
    workload's kind) with injected noise, all in one launch (float64, the
    default seam-window solve): every task equals the oracle's emd_1d of its
    own perturbed input -- identical knot counts in every sift, IMFs within
    1e-9 of max|x| (emd_ref.py:108-156)."""
    from oracle import emd_oracle as O
    from test_gpu_parity import engine_log, max_imf_err, oracle_log, raw_run

    lengths = [int(round(v)) for v in np.geomspace(4096, 65536, 8)]
    rng = np.random.default_rng(11)
    rows = []
    for i, n in enumerate(lengths):
        x = signals.harmonic_clicks(n, seed=1000 + i)
        rows.append(x + 0.2 * np.std(x) * rng.standard_normal(n))
    res = raw_run(None, x=np.concatenate(rows), lengths=lengths, trial_count=1,
                  noise_mode=L.EEMD_NOISE_PREPERTURBED, tau=0.0, max_sifts=10, max_imf=10, exact=False)
    for t, row in enumerate(rows):
        imfs, _, st = O.emd_1d(row, tau=0.0, max_sifts=10, max_imf=10, record_knots=True)
        assert int(res["nmode"][t]) == st["n_modes"]
        assert engine_log(res, t) == oracle_log(st), t
        err = max_imf_err(res["imfs"][t][:st["n_modes"]], imfs, np.abs(row).max())
        assert err <= 1e-9, (t, err)
