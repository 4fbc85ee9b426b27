"""The oracle against the reference's own emd_ref.emd_1d (installed unchanged
in baseline/_ref by baseline/install_reference.py) on the signals the GPU
edge tests use: the shortest and ragged lengths, flat, ramp and plateau
signals, natural and mirror ends.  Bit-for-bit: the same IMFs, residual,
mode and sift counts (emd_ref.py:108-156).  Skipped when the reference is
not installed."""
import importlib.util
from pathlib import Path

import numpy as np
import pytest

from oracle import emd_oracle as O
from test_gpu_edges import edge_rows

REF = Path(__file__).resolve().parents[1] / "baseline" / "_ref" / "emd_ref.py"


@pytest.fixture(scope="module")
def ref():
    if not REF.exists():
        pytest.skip("the reference is not installed in baseline/_ref "
                    "(python baseline/install_reference.py <reference checkout>)")
    spec = importlib.util.spec_from_file_location("_reference_emd_ref", REF)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def flat_and_plateau_rows():
    t = np.arange(3000, dtype=float)
    return [np.zeros(1000), np.linspace(-1.0, 2.0, 777),
            np.clip(1.5 * np.sin(2 * np.pi * t / 97.0), -1, 1) + 0.3 * np.sin(2 * np.pi * t / 11.0),
            np.round(64 * (np.sin(2 * np.pi * t / 40.0) + 0.4 * np.sin(2 * np.pi * t / 7.0))) / 64]


@pytest.mark.parametrize("end", ["natural", "mirror"])
@pytest.mark.parametrize("rows", ["edge5", "edge6", "flat"])
def test_oracle_equals_reference_at_the_edges(ref, end, rows):
    xs = {"edge5": lambda: edge_rows(5), "edge6": lambda: edge_rows(6), "flat": flat_and_plateau_rows}[rows]()
    for x in xs:
        ri, rr, rs = ref.emd_1d(x, tau=0.25, max_sifts=50, max_imf=10, end=end)
        oi, orr, os_ = O.emd_1d(x, tau=0.25, max_sifts=50, max_imf=10, end=end)
        ri = np.asarray(ri, dtype=float).reshape(-1, len(x))
        oi = np.asarray(oi, dtype=float).reshape(-1, len(x))
        assert ri.shape == oi.shape, len(x)
        assert np.array_equal(ri, oi) and np.array_equal(rr, orr), len(x)
        assert (rs["n_modes"], rs["total_sifts"]) == (os_["n_modes"], os_["total_sifts"]), len(x)
        assert list(rs["per_mode_sifts"]) == list(os_["per_mode_sifts"]), len(x)
