"""Parity and size-independent properties at the benchmark workloads' full sizes.

* the 2^22-sample AM/FM signal (the amfm4m workload, float64): the first sift
  against the oracle (knot counts identical, IMF within the tolerances of
  test_gpu_parity), launch-shape invariance (bit-identical results for 4 and
  8 CTAs per task), and the per-trial identity sum(IMFs) + residual = input
  of two noisy trials carried through every IMF;
* the 48 000-sample harmonic+clicks signal (the harmonic48k workload, float64
  storage so that the knots are comparable): two noisy trials of 8 IMFs x 10
  fixed sifts against the oracle, knot counts of every sift included.
"""
import numpy as np
import pytest

from eemd4cuda_b200 import emd_par as M
from eemd4cuda_b200 import signals
from oracle import emd_oracle as O
from test_gpu_parity import engine_log, max_imf_err, oracle_log, raw_run

pytestmark = pytest.mark.gpu

N_AMFM = 1 << 22


@pytest.fixture(scope="module")
def amfm():
    return signals.amfm_long(N_AMFM, seed=2)


@pytest.mark.parametrize("exact", [True, False])
def test_amfm_first_sift_fullsize(amfm, exact):
    """One sift of 4 194 304 samples (about 1.27 M knots per envelope)."""
    cfg = None if exact else M.EngineConfig(halo=30)
    res = raw_run(amfm[None, :], tau=0.0, max_sifts=1, max_imf=1, exact=exact, config=cfg)
    imfs, _, st = O.emd_1d(amfm, tau=0.0, max_sifts=1, max_imf=1, record_knots=True)
    assert engine_log(res, 0) == oracle_log(st)
    err = max_imf_err(res["imfs"][0][:1], imfs, np.abs(amfm).max())
    assert err <= (1e-12 if exact else 1e-9), err


def test_amfm_launch_shape_invariance_fullsize(amfm):
    """Fixed sifts: the knot lists, the solve windows and every sample's
    arithmetic are independent of how many CTAs share the signal."""
    kw = dict(tau=0.0, max_sifts=2, max_imf=2, exact=False)
    a = raw_run(amfm[None, :], config=M.EngineConfig(halo=30, cluster_size=4), **kw)
    b = raw_run(amfm[None, :], config=M.EngineConfig(halo=30, cluster_size=8), **kw)
    assert a["nmode"].tolist() == b["nmode"].tolist()
    assert np.array_equal(a["knot_log"], b["knot_log"])
    for u, v in zip(a["imfs"][0], b["imfs"][0]):
        assert np.array_equal(u, v)
    assert np.array_equal(a["resid"][0], b["resid"][0])


def test_amfm_trial_reconstruction_fullsize(amfm):
    """Every trial's modes and residual add back to that trial's input (the
    amfm4m settings: tau 0.2, up to 20 sifts, 12 IMFs, seam halo 30)."""
    rng = np.random.default_rng(5)
    X = amfm[None, :] + 0.2 * np.std(amfm) * rng.standard_normal((2, N_AMFM))
    res = raw_run(X, tau=0.2, max_sifts=20, max_imf=12, exact=False, config=M.EngineConfig(halo=30))
    for e in range(2):
        m = int(res["nmode"][e])
        assert 6 <= m <= 12
        rec = res["imfs"][e][:m].sum(axis=0) + res["resid"][e]
        assert np.max(np.abs(rec - X[e])) <= 1e-12 * np.abs(X[e]).max()


def test_harmonic_trials_fullsize():
    """Two noisy trials of the 48 000-sample workload, 8 IMFs x 10 sifts."""
    x = signals.harmonic_clicks(48000, seed=1)
    rng = np.random.default_rng(11)
    X = x[None, :] + 0.2 * np.std(x) * rng.standard_normal((2, len(x)))
    res = raw_run(X, tau=0.0, max_sifts=10, max_imf=8, exact=False)
    for e in range(2):
        imfs, _, st = O.emd_1d(X[e], tau=0.0, max_sifts=10, max_imf=8, record_knots=True)
        assert int(res["nmode"][e]) == st["n_modes"]
        assert engine_log(res, e) == oracle_log(st)
        err = max_imf_err(res["imfs"][e][:st["n_modes"]], imfs, np.abs(X[e]).max())
        assert err <= 1e-9, err
