"""CEEMDAN on the GPU engine against the reference's own results
(tests/golden/ceemdan_cases.npz, made by emd_ref.ceemdan) and the CPU oracle."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import emd_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from eemd4cuda_b200.ceemdan import ceemdan  # noqa: E402

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
def test_exact_ceemdan_equals_reference(golden, name):
    x = golden[f"{name}_x"]
    c, r, st = ceemdan(x, exact=True, **params(golden, name))
    assert st["noise_modes"] == golden[f"{name}_noise_modes"].tolist()
    assert st["n_imfs"] == golden[f"{name}_c"].shape[0]
    scale = np.abs(x).max()
    assert np.max(np.abs(c - golden[f"{name}_c"])) <= 1e-9 * scale
    assert np.max(np.abs(r - golden[f"{name}_r"])) <= 1e-9 * scale
    # per-stage sift counts against the oracle's
    _, _, ost = O.ceemdan(x, **params(golden, name))
    assert st["stage_sifts"] == ost["stage_sifts"]


@pytest.mark.parametrize("name", CASES)
def test_fast_ceemdan_is_complete_and_close(golden, name):
    x = golden[f"{name}_x"]
    c, r, st = ceemdan(x, **params(golden, name))
    scale = np.abs(x).max()
    assert np.max(np.abs(x - c.sum(axis=0) - r)) <= 1e-12 * scale
    assert st["noise_modes"] == golden[f"{name}_noise_modes"].tolist()
    if st["n_imfs"] == golden[f"{name}_c"].shape[0]:
        assert np.max(np.abs(c - golden[f"{name}_c"])) <= 1e-6 * scale


def test_ceemdan_48k_staircase_properties():
    from eemd4cuda_b200 import signals
    x = signals.harmonic_clicks(48000, seed=1)
    c, r, st = ceemdan(x, E=32, eps=0.2, seed=0, tau=0.25, max_sifts=50)
    assert np.max(np.abs(x - c.sum(axis=0) - r)) <= 1e-12 * np.abs(x).max()
    # the staircase ends after stage max(noise modes) unless the residual vanished first
    assert st["n_imfs"] <= max(st["noise_modes"]) + 1
    assert all(len(s) == 32 for s in st["stage_sifts"])


def test_philox_noise_ceemdan():
    """noise='philox': W drawn on the device; the staircase is complete and
    deterministic, and W is standard normal."""
    from eemd4cuda_b200 import _lib as L
    from eemd4cuda_b200 import signals
    W = torch.empty((16, 20000), dtype=torch.float64, device="cuda")
    L.philox_normals(5, 0, 0, 16, 20000, W)
    w = W.cpu().numpy()
    assert abs(w.mean()) < 0.01 and abs(w.std() - 1.0) < 0.01
    W2 = torch.empty_like(W)
    L.philox_normals(5, 0, 0, 16, 20000, W2)
    assert torch.equal(W, W2)
    L.philox_normals(5, 0, 3, 2, 20000, W2[:2])
    assert torch.equal(W2[:2], W[3:5])  # keyed by the absolute trial
    x = signals.harmonic_clicks(8000, seed=2, fs=8000.0)
    a = ceemdan(x, E=16, seed=5, noise="philox")
    b = ceemdan(x, E=16, seed=5, noise="philox")
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    c, r, st = a
    assert np.max(np.abs(x - c.sum(axis=0) - r)) <= 1e-12 * np.abs(x).max()
    assert st["n_imfs"] <= max(st["noise_modes"]) + 1
