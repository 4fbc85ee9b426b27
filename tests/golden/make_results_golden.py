"""Generate the result-format fixtures from the reference implementation itself.

    python tests/golden/make_results_golden.py <reference checkout>

Runs the reference's audio_eemd/report.py write_imfs_npz (loaded as a module
under a bare package stand-in, so the package's audio dependencies are not
imported) and emd_par.EMDResult.save on a small decomposition, and copies
the two files to tests/golden/ref_imfs.npz and tests/golden/ref_emdresult.npz.
Nothing under tests/ reads the reference at test time.
"""
from __future__ import annotations

import importlib.util
import shutil
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


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


def main(ref_dir: str):
    pkg = types.ModuleType("audio_eemd")
    pkg.__path__ = [str(Path(ref_dir) / "audio_eemd")]
    pkg.__version__ = "0"
    sys.modules["audio_eemd"] = pkg
    spec = importlib.util.spec_from_file_location("audio_eemd.report", Path(ref_dir) / "audio_eemd" / "report.py")
    rep = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rep)
    sys.path.insert(0, ref_dir)
    import emd_par

    x, t, imfs, residual, stats = case()
    with tempfile.TemporaryDirectory() as d:
        p = rep.write_imfs_npz(Path(d), x, t, imfs, residual, 3, stats)
        shutil.copy(p, HERE / "ref_imfs.npz")
        r = emd_par.EMDResult(imfs=imfs, residual=residual, n_modes=3, stats=stats)
        r.save(str(Path(d) / "r.npz"))
        shutil.copy(Path(d) / "r.npz", HERE / "ref_emdresult.npz")
    print("written")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
