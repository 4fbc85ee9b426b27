"""Edge lengths in one launch against the oracle: signals from the minimum
length (8 samples) through lengths on either side of the 32-sample segment
granule up to a few thousand samples, every task checked against the
oracle's emd_1d of the same input (emd_ref.py:108-156)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
pytest.importorskip("torch")

from eemd4cuda_b200 import _lib as L  # noqa: E402

LENGTHS = [8, 9, 13, 31, 32, 33, 64, 95, 257, 1000, 2049, 4097]


def edge_rows(seed=5):
    """Two tones and white noise per length: extrema at every scale, and at
    the shortest lengths fewer extrema than an IMF needs."""
    rng = np.random.default_rng(seed)
    rows = []
    for n in LENGTHS:
        t = np.arange(n, dtype=float)
        rows.append(np.sin(2 * np.pi * t / 17.0) + 0.5 * np.sin(2 * np.pi * t / 5.3)
                    + 0.3 * rng.standard_normal(n))
    return rows


@pytest.mark.parametrize("end", ["natural", "mirror"])
@pytest.mark.parametrize("exact", [True, False])
def test_short_and_ragged_lengths_against_oracle(end, exact):
    """Mode count, the knot counts of every sift and the IMFs and residual of
    every task equal the oracle's (IMFs within 1e-12 of max|x| in exact mode,
    1e-9 with the seam-window solve).  Exact mode runs the SD stop rule
    (tau 0.25, at most 50 sifts); the fast solve runs fixed sift counts
    (tau 0, 10 sifts), where no SD comparison can fall either way."""
    from oracle import emd_oracle as O
    from test_gpu_parity import engine_log, max_imf_err, oracle_log, raw_run

    tau, max_sifts = (0.25, 50) if exact else (0.0, 10)
    tol = 1e-12 if exact else 1e-9
    rows = edge_rows()
    res = raw_run(None, x=np.concatenate(rows), lengths=LENGTHS, trial_count=1,
                  noise_mode=L.EEMD_NOISE_PREPERTURBED, tau=tau, max_sifts=max_sifts, max_imf=10,
                  exact=exact, end=end)
    for t, row in enumerate(rows):
        imfs, resid, st = O.emd_1d(row, tau=tau, max_sifts=max_sifts, max_imf=10, end=end,
                                   record_knots=True)
        scale = np.abs(row).max()
        assert int(res["nmode"][t]) == st["n_modes"], (LENGTHS[t], int(res["nmode"][t]), st["n_modes"])
        assert engine_log(res, t) == oracle_log(st), LENGTHS[t]
        err = max_imf_err(res["imfs"][t][:st["n_modes"]], imfs, scale)
        assert err <= tol, (LENGTHS[t], err)
        assert np.max(np.abs(res["resid"][t] - resid)) <= tol * scale * max(1, st["n_modes"]), LENGTHS[t]
