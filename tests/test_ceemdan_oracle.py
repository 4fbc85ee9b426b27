"""The CEEMDAN restatement in oracle/emd_oracle.py against fixtures made by
the reference's own emd_ref.ceemdan (tests/golden/make_ceemdan_golden.py)."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import emd_oracle as O

CASES = ["a", "b", "c"]


@pytest.fixture(scope="module")
def golden():
    d = np.load(GOLDEN / "ceemdan_cases.npz")
    return {k: d[k] for k in d.files}


def params(g, name):
    N, E, eps, seed, tau, ms, end = g[f"{name}_params"]
    return dict(E=int(E), eps=float(eps), seed=int(seed), tau=float(tau), max_sifts=int(ms),
                end="natural" if end == 0 else "mirror")


@pytest.mark.parametrize("name", CASES)
def test_oracle_ceemdan_matches_reference(golden, name):
    x = golden[f"{name}_x"]
    c, r, st = O.ceemdan(x, **params(golden, name))
    assert st["n_imfs"] == golden[f"{name}_c"].shape[0]
    assert st["noise_modes"] == golden[f"{name}_noise_modes"].tolist()
    scale = np.abs(x).max()
    assert np.max(np.abs(c - golden[f"{name}_c"])) <= 1e-12 * scale
    assert np.max(np.abs(r - golden[f"{name}_r"])) <= 1e-12 * scale
    # the decomposition is complete
    assert np.max(np.abs(x - c.sum(axis=0) - r)) <= 1e-12 * scale
