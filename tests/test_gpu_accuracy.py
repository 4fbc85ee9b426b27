"""Accuracy of the bench workload's arithmetic against the float64 CPU oracle.

The 48 kHz bench workload (harmonic tone + pink noise + clicks, N = 48 000,
8 IMFs x 10 fixed sifts) runs with float32 storage: samples, IMFs and the
envelopes' interval records are float32 and the spline evaluation, the mean
envelope and the subtraction run in float32; only the tridiagonal
elimination is float64.  The reference computes everything in float64
(emd_ref.py:108-156).  Here the oracle (float64 throughout) runs on the very
same trial inputs -- the float32-rounded x + noise rows -- so every
difference measured is the engine's own arithmetic.

Stated bounds (relative L2 error per IMF, ||imf - imf_oracle|| / ||imf_oracle||):
  float32 storage, fast solve : IMF k <= F32_IMF_BOUNDS[k] on every trial, and
                                <= F32_STACK_BOUND for the whole stack
                                (||IMFs - IMFs_oracle||_F / ||x||)
  float64 storage, fast solve : <= 1e-9 on every IMF, and every sift's knot
                                counts identical
The first sift of every trial sees identical input values, so its knot
counts must be identical.  Later sifts may differ where two neighbouring
samples are closer than float32 rounding: the strict-extremum test then
decides differently from the float64 one, the envelope changes around that
knot, and the difference is carried into every later IMF (the sift count per
IMF is fixed, so the mode count never changes).  The first IMFs therefore
agree to float32 rounding (measured 2e-7 - 1e-6 on IMFs 1-3 of these
inputs); later IMFs differ from the float64 ones wherever such a decision
flipped, by an amount set by the flip, not by rounding (measured up to
2e-3 / 0.11 / 0.11 / 0.23 / 0.35 on IMFs 4-8 and 3.7e-2 on the stack here,
5.5e-4 already on IMF 3 of another input).  The bounds for IMFs 1-2 are
accuracy claims; those for later IMFs only say that no trial diverges
further than a flip does.
"""
import numpy as np
import pytest

from eemd4cuda_b200 import signals
from oracle import emd_oracle as O
from test_gpu_parity import raw_run

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N = 48000
TRIALS = 4
F32_IMF_BOUNDS = [1e-5, 1e-5, 1e-2, 5e-2, 3e-1, 5e-1, 1.0, 1.0]
F32_STACK_BOUND = 2e-1


def _trial_inputs(dtype):
    """x (float32-rounded, as the bench uploads it) + 0.2*std(x) white noise,
    rounded to the storage type: the rows both sides decompose."""
    x = signals.harmonic_clicks(N, seed=1).astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(7)
    noise = 0.2 * np.std(x) * rng.standard_normal((TRIALS, N))
    return (x[None, :] + noise).astype(dtype)


def _accuracy(res, X):
    """Per-trial, per-IMF relative L2 errors against the oracle, the stack
    error, and the knot-count agreement of the sifts."""
    rel, stack, same_sifts, total_sifts, first_ok = [], [], 0, 0, True
    for e in range(X.shape[0]):
        xo = X[e].astype(np.float64)
        imfs, _, st = O.emd_1d(xo, tau=0.0, max_sifts=10, max_imf=8, record_knots=True)
        assert int(res["nmode"][e]) == st["n_modes"] == 8
        g = res["imfs"][e][:8]
        rel.append([float(np.linalg.norm(g[k] - imfs[k]) / np.linalg.norm(imfs[k])) for k in range(8)])
        stack.append(float(np.linalg.norm(g - imfs) / np.linalg.norm(xo)))
        for m, mode in enumerate(st["knot_log"]):
            for k, (a, b) in enumerate(mode):
                total_sifts += 1
                same = res["knot_log"][e, m, k].tolist() == [a, b]
                same_sifts += int(same)
                if m == 0 and k == 0:
                    first_ok = first_ok and same
    return np.array(rel), np.array(stack), same_sifts, total_sifts, first_ok


def test_float32_storage_against_float64_oracle():
    X = _trial_inputs(np.float32)
    res = raw_run(X, tau=0.0, max_sifts=10, max_imf=8, exact=False, dtype=np.float32)
    rel, stack, same, total, first_ok = _accuracy(res, X)
    print(f"float32 storage vs float64 oracle: max rel L2 per IMF {rel.max(axis=0)}, "
          f"stack {stack.max():.3e}, sifts with identical knot counts {same}/{total}")
    assert first_ok
    assert np.all(rel.max(axis=0) <= np.array(F32_IMF_BOUNDS)), rel.max(axis=0)
    assert stack.max() <= F32_STACK_BOUND, stack
    # the per-trial partition of unity holds to float32 rounding
    for e in range(TRIALS):
        recon = res["imfs"][e][:8].sum(axis=0) + res["resid"][e] - X[e].astype(np.float64)
        assert np.max(np.abs(recon)) <= 1e-5 * np.abs(X[e]).max()


def test_float64_storage_against_float64_oracle():
    X = _trial_inputs(np.float64)
    res = raw_run(X, tau=0.0, max_sifts=10, max_imf=8, exact=False, dtype=np.float64)
    rel, stack, same, total, first_ok = _accuracy(res, X)
    print(f"float64 storage vs float64 oracle: max rel L2 per IMF {rel.max(axis=0)}, "
          f"stack {stack.max():.3e}, sifts with identical knot counts {same}/{total}")
    assert first_ok
    assert same == total
    assert rel.max() <= 1e-9, rel.max(axis=0)
