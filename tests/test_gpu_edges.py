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


def test_numba_rules_at_short_and_ragged_lengths():
    """The numba kernel's stop rules (emd_gpu.py:152-274: an IMF also ends
    with fewer than 2 maxima or minima; SD = sum(m^2)/sum(h^2)) on the same
    edge lengths: mode counts, knot counts and IMFs equal the oracle's."""
    from oracle import emd_oracle as O
    from test_gpu_parity import engine_log, max_imf_err, oracle_log, raw_run

    rows = edge_rows(seed=6)
    res = raw_run(None, x=np.concatenate(rows), lengths=LENGTHS, trial_count=1,
                  noise_mode=L.EEMD_NOISE_PREPERTURBED, tau=0.25, max_sifts=50, max_imf=10,
                  rules="numba", exact=True)
    for t, row in enumerate(rows):
        imfs, _, st = O.emd_1d(row, tau=0.25, max_sifts=50, max_imf=10, rules="numba", record_knots=True)
        assert int(res["nmode"][t]) == st["n_modes"], LENGTHS[t]
        assert engine_log(res, t) == oracle_log(st), LENGTHS[t]
        assert max_imf_err(res["imfs"][t][:st["n_modes"]], imfs, np.abs(row).max()) <= 1e-12, LENGTHS[t]


def test_public_calls_at_short_and_ragged_lengths():
    """decompose and decompose_many (E = 1) on the edge lengths: the same
    modes, a (0, N) IMF array where the signal has too few extrema, and
    IMFs + residual = input."""
    from eemd4cuda_b200 import emd_par as M

    rows = edge_rows(seed=7)
    many = M.decompose_many(rows, E=1, tau=0.25, max_sifts=50, max_imf=10, exact=True)
    for x, r in zip(rows, many):
        one = M.decompose(x, E=1, tau=0.25, max_sifts=50, max_imf=10, exact=True)
        assert r.n_modes == one.n_modes and r.imfs.shape == (r.n_modes, len(x))
        assert np.array_equal(r.imfs, one.imfs)
        assert np.max(np.abs(x - one.imfs.sum(axis=0) - one.residual)) <= 1e-12 * np.abs(x).max()
    assert many[LENGTHS.index(9)].n_modes == 0


def test_flat_ramp_and_plateau_signals_against_oracle():
    """Signals without extrema (all zeros, a straight ramp: no IMF, the
    residual is the input) and signals with equal neighbouring samples (a
    clipped tone, a tone quantised to 1/64: strict extrema only, so plateaus
    give no knots), in one launch, exact mode: the oracle's mode counts, knot
    counts and IMFs."""
    from oracle import emd_oracle as O
    from test_gpu_parity import engine_log, max_imf_err, oracle_log, raw_run

    t = np.arange(3000, dtype=float)
    rows = [np.zeros(1000), np.linspace(-1.0, 2.0, 777),
            np.clip(1.5 * np.sin(2 * np.pi * t / 97.0), -1, 1) + 0.3 * np.sin(2 * np.pi * t / 11.0),
            np.round(64 * (np.sin(2 * np.pi * t / 40.0) + 0.4 * np.sin(2 * np.pi * t / 7.0))) / 64]
    lengths = [len(r) for r in rows]
    res = raw_run(None, x=np.concatenate(rows), lengths=lengths, trial_count=1,
                  noise_mode=L.EEMD_NOISE_PREPERTURBED, tau=0.25, max_sifts=50, max_imf=10, exact=True)
    for k, row in enumerate(rows):
        imfs, resid, st = O.emd_1d(row, tau=0.25, max_sifts=50, max_imf=10, record_knots=True)
        assert int(res["nmode"][k]) == st["n_modes"], k
        assert engine_log(res, k) == oracle_log(st), k
        scale = max(np.abs(row).max(), 1.0)
        assert max_imf_err(res["imfs"][k][:st["n_modes"]], imfs, scale) <= 1e-12, k
        assert np.max(np.abs(res["resid"][k] - resid)) <= 1e-12 * scale * max(1, st["n_modes"]), k
    assert int(res["nmode"][0]) == 0 and int(res["nmode"][1]) == 0
    assert np.array_equal(res["resid"][1], rows[1])
