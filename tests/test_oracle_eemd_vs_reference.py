"""The oracle's EEMD (per-trial default_rng noise of the reference's CPU path,
trial-ordered per-mode means) against the reference's own
emd_par.decompose(method='cpu') (emd_par.py:112-154), installed unchanged in
baseline/_ref by baseline/install_reference.py: bit-for-bit the same means
and residual.  Skipped when the reference is not installed."""
import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import emd_oracle as O

REF = Path(__file__).resolve().parents[1] / "baseline" / "_ref"


@pytest.fixture(scope="module")
def ref_emd_par():
    if not (REF / "emd_par.py").exists():
        pytest.skip("the reference is not installed in baseline/_ref "
                    "(python baseline/install_reference.py <reference checkout>)")
    sys.path.insert(0, str(REF))  # its `import emd_ref`
    try:
        name = "_reference_emd_par"
        spec = importlib.util.spec_from_file_location(name, REF / "emd_par.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod  # dataclasses resolve the module while the class body runs
        spec.loader.exec_module(mod)
        yield mod
    finally:
        sys.path.remove(str(REF))
        sys.modules.pop("_reference_emd_par", None)


@pytest.mark.parametrize("N,E,seed,end", [(2000, 4, 3, "natural"), (3001, 6, 11, "mirror"), (777, 5, 0, "natural")])
def test_oracle_eemd_equals_reference_cpu_path(ref_emd_par, N, E, seed, end):
    from eemd4cuda_b200 import signals

    x = signals.harmonic_clicks(N, seed=seed, fs=8000.0)
    r = ref_emd_par.decompose(x, method="cpu", E=E, eps=0.2, tau=0.25, max_sifts=50, max_imf=-1, end=end,
                              seed=seed, parallel=False)
    X = x[None, :] + O.noise_cpu_stream(x, E, 0.2, seed)
    avg, resid, _ = O.eemd(x, X, tau=0.25, max_sifts=50, max_imf=-1, end=end)
    assert r.n_modes == avg.shape[0]
    assert np.array_equal(r.imfs, avg) and np.array_equal(r.residual, resid)
