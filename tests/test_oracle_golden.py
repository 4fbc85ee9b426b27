"""Pin the CPU oracle against the reference's own outputs (tests/golden/).

The fixtures were produced by the reference implementation (emd_ref.py, its
DSBT host mirror and its numba kernel under the CUDA simulator) by
tests/golden/make_golden.py.  These tests need no GPU.
"""
import numpy as np
import pytest

from conftest import checksum_close
from oracle import emd_oracle as O
from eemd4cuda_b200 import signals


def test_sweep_generator_matches_reference(known):
    assert known["sweep_identical_to_refsignal"]


def test_config_A_known_answer(known, sweep):
    """ref[:110250], E=1: 9 modes, 26 sifts (phase3_gates.log:2)."""
    imfs, resid, st = O.emd_1d(sweep[:110250], tau=0.25, max_sifts=50, max_imf=16)
    A = known["A"]
    assert st["n_modes"] == A["n_modes"] == 9
    assert st["total_sifts"] == A["total_sifts"] == 26
    assert st["per_mode_sifts"] == A["per_mode_sifts"]
    for m, ck in zip(imfs, A["imf"]):
        ok, err = checksum_close(m, ck)
        assert ok, err
    ok, err = checksum_close(resid, A["resid"])
    assert ok, err


def test_config_B_known_answer(known, sweep):
    """8 seed-7 trials: nmode [10]*8, nsift [22,22,23,21,24,23,23,29]."""
    x = sweep[:110250]
    rng = np.random.default_rng(7)
    X = x[None, :] + 0.2 * np.std(x) * rng.standard_normal((8, len(x)))
    B = known["B"]
    for e in range(8):
        imfs, _, st = O.emd_1d(X[e], tau=0.25, max_sifts=50, max_imf=16)
        assert st["n_modes"] == B["n_modes"][e]
        assert st["total_sifts"] == B["total_sifts"][e]
        assert st["per_mode_sifts"] == B["per_mode_sifts"][e]
        assert checksum_close(imfs[0], B["imf0"][e])[0]
        assert checksum_close(imfs[-1], B["imf_last"][e])[0]
    assert B["total_sifts"] == [22, 22, 23, 21, 24, 23, 23, 29]


def test_plain_8k_mirror_bit_exact(known, small):
    x = signals.plain_emd_8k()
    assert np.array_equal(x, small["plain8k_x"])
    imfs, resid, st = O.emd_1d(x, tau=0.2, max_sifts=10, max_imf=10, end="mirror")
    K = known["plain8k_mirror"]
    assert st["n_modes"] == K["n_modes"] == 6
    assert st["per_mode_sifts"] == K["per_mode_sifts"]
    assert np.array_equal(np.array(imfs), small["plain8k_imfs"])
    assert np.array_equal(resid, small["plain8k_resid"])


@pytest.mark.parametrize("end", ["natural", "mirror"])
def test_chirp2048(known, small, end):
    imfs, resid, st = O.emd_1d(small["a1_x"], tau=0.25, max_sifts=50, end=end)
    K = known[f"chirp2048_{end}"]
    assert st["n_modes"] == K["n_modes"]
    assert st["per_mode_sifts"] == K["per_mode_sifts"]
    assert np.array_equal(np.array(imfs), small[f"chirp2048_{end}_imfs"])


def test_one_sift(small):
    h1 = O.one_sift(small["a1_x"])
    assert np.array_equal(h1, small["a1_h1"])


def test_pathological_chirp(known):
    x = signals.modulated_chirp()
    imfs, _, st = O.emd_1d(x, tau=0.25, max_sifts=50, max_imf=16)
    G = known["G8"]
    assert st["n_modes"] == G["n_modes"]
    assert st["total_sifts"] == G["total_sifts"]
    for m, ck in zip(imfs, G["imf"]):
        assert checksum_close(m, ck)[0]


def test_two_tones_stage_fixture(known):
    x, _ = signals.two_tones()
    _, _, st = O.emd_1d(x, tau=0.25, max_sifts=50)
    assert st["n_modes"] == known["two_tones"]["n_modes"]
    assert st["per_mode_sifts"] == known["two_tones"]["per_mode_sifts"]


def test_numba_rules_match_simulated_reference_kernel(known, small):
    """Oracle rules='numba' vs the reference numba kernel (emd_gpu.py) run under
    numba's CUDA simulator: same sift/mode counts, IMFs to 1e-13."""
    K = known["numba_sim"]
    X = small["numba_X"]
    out = small["numba_out"]
    for e in range(X.shape[0]):
        imfs, _, st = O.emd_1d(X[e], tau=K["tau"], max_sifts=K["max_sifts"], max_imf=K["maximf"],
                               rules="numba")
        assert st["n_modes"] == K["nmode"][e]
        assert st["total_sifts"] == K["nsift"][e]
        for m in range(st["n_modes"]):
            assert np.max(np.abs(imfs[m] - out[e, m])) <= 1e-13


@pytest.mark.parametrize("kind", ["uniform", "cv15"])
def test_dsbt_mirror(small, kind):
    """Seam-window Thomas (B=250, S=30) equals the reference's fixed host
    mirror bit for bit and the exact Thomas to <= 1e-15 relative (gate U1)."""
    tm = small[f"dsbt_{kind}_tm"].astype(float)
    ym = small[f"dsbt_{kind}_ym"]
    dg, lo, up, r = O.spline_system(tm, ym)
    x = O.dsbt_solve(dg, lo, up, r, B=250, S=30)
    assert np.array_equal(x, small[f"dsbt_{kind}_x"])
    ex = O.thomas(dg, lo, up, r)
    assert np.array_equal(ex, small[f"dsbt_{kind}_exact"])
    assert np.max(np.abs(x - ex)) / np.max(np.abs(ex)) <= 1e-15


def _scan_cases():
    rng = np.random.default_rng(0)
    cases = {"random": rng.standard_normal(5000)}
    x = rng.standard_normal(4000)
    x[100:110] = x[100]
    x[200:260] = x[200]
    cases["flat_runs"] = x
    x = rng.standard_normal(4000)
    x[500:505] = 99.0
    cases["plateau"] = x
    x = np.linspace(0, 1, 1000)
    x[500] = 5.0
    cases["single_max"] = x
    x = np.linspace(0, 1, 1000)
    x[500] = -5.0
    cases["single_min"] = x
    cases["constant"] = np.ones(500)
    cases["monotone"] = np.linspace(-3, 3, 2000)
    cases["alternating"] = (np.arange(1000) % 2) * 2.0 - 1.0
    return cases


@pytest.mark.parametrize("name", list(_scan_cases().keys()))
def test_tile_scan_equals_serial(name):
    """Gate U2: tile-ordered compaction is bit-identical to the serial scan."""
    x = _scan_cases()[name]
    imax, imin = O.extrema(x)
    for tile in (32, 128, 1024):
        assert np.array_equal(O.scan_tiles(x, True, tile), imax)
        assert np.array_equal(O.scan_tiles(x, False, tile), imin)


def test_ensemble_mean_order():
    """Masked per-mode mean in trial order, residual x - sum(mean)."""
    x = np.arange(5.0)
    a = [[np.ones(5), 2 * np.ones(5)], [3 * np.ones(5)]]
    avg, resid, cnt = O.ensemble_mean(x, a)
    assert np.array_equal(cnt, [2, 1])
    assert np.array_equal(avg[0], 2 * np.ones(5))
    assert np.array_equal(avg[1], 2 * np.ones(5))
    assert np.array_equal(resid, x - 4)
