"""Result files in the reference's formats: imfs.npz (audio_eemd/report.py:177-194)
and EMDResult.save (emd_par.py:84-97), against files the reference itself wrote
(tests/golden/make_results_golden.py)."""
import numpy as np

from conftest import GOLDEN
from eemd4cuda_b200 import results


def case():
    rng = np.random.default_rng(0)
    N = 64
    x = rng.standard_normal(N)
    imfs = rng.standard_normal((3, N))
    residual = x - imfs.sum(axis=0)
    t = np.arange(N) / 8000.0
    stats = dict(method="gpu", E=8, total_sifts=31, per_mode_sifts=[10, 12, 9], gpu_time_s=0.25,
                 max_imf_reached=False, x=x, n_workers=1)
    return x, t, imfs, residual, stats


def same_npz(a, b):
    da, db = np.load(a), np.load(b)
    assert sorted(da.files) == sorted(db.files)
    for k in da.files:
        assert da[k].dtype == db[k].dtype, k
        assert da[k].shape == db[k].shape, k
        assert np.array_equal(da[k], db[k]), k


def test_imfs_npz_matches_the_reference_file(tmp_path):
    x, t, imfs, residual, stats = case()
    p = results.write_imfs_npz(tmp_path, x, t, imfs, residual, 3, stats)
    same_npz(p, GOLDEN / "ref_imfs.npz")


def test_emdresult_file_matches_the_reference_file(tmp_path):
    x, t, imfs, residual, stats = case()
    results.save_result(tmp_path / "r.npz", imfs, residual, 3, stats)
    same_npz(tmp_path / "r.npz", GOLDEN / "ref_emdresult.npz")
    from eemd4cuda_b200.emd_par import EMDResult
    r = EMDResult.load(str(GOLDEN / "ref_emdresult.npz"))
    assert r.n_modes == 3 and np.array_equal(r.imfs, imfs) and int(r.stats["total_sifts"]) == 31
