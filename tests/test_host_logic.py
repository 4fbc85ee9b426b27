"""Host-side logic of the drop-in API (no GPU needed): validation and error
mapping (emd_par.py:282-286; the reference's own eemd_stage.py:66-77 on top),
result container, reference noise streams, IMF slot bound."""
import numpy as np
import pytest

from eemd4cuda_b200 import emd_par as M
import ref_stage
from oracle import emd_oracle as O


def test_bad_input_raises_value_error():
    with pytest.raises(ValueError):
        M.decompose(np.ones(5))
    with pytest.raises(ValueError):
        M.decompose(np.ones((4, 10)))
    with pytest.raises(ValueError):
        M.decompose(np.ones(100), method="cpu")
    with pytest.raises(ValueError):
        M.decompose(np.ones(100), method="quantum")


def test_stage_maps_bad_input(monkeypatch):
    """audio_eemd/tests/test_eemd_stage.py:65-69 through the reference's own
    stage adapter on the compat module: np.ones(5) -> eemd.bad_input, and the
    CPU method this engine does not offer -> eemd.bad_input."""
    stage = ref_stage.load(monkeypatch)
    with pytest.raises(stage.EEMDError) as ei:
        stage.run_eemd(np.ones(5), method="gpu", E=1)
    assert ei.value.code == "eemd.bad_input"
    with pytest.raises(stage.EEMDError) as ei:
        stage.run_eemd(np.ones(100), method="cpu", E=1)
    assert ei.value.code == "eemd.bad_input"


def test_gpu_eemd_full_guard():
    """test_emd_gpu.py A5: 1-D input with E>1 raises ValueError."""
    with pytest.raises(ValueError):
        M.gpu_eemd_full(np.ones(1000), E=4)


def test_emdresult_roundtrip(tmp_path):
    x = np.linspace(0, 1, 50)
    r = M.EMDResult(imfs=np.stack([x, 2 * x]), residual=-2 * x, n_modes=2,
                    stats={"method": "gpu", "E": 4, "gpu_time_s": 0.5, "x": x})
    assert r.recon_error() == pytest.approx(0.0, abs=1e-15)
    r.save(str(tmp_path / "r.npz"))
    q = M.EMDResult.load(str(tmp_path / "r.npz"))
    assert np.array_equal(q.imfs, r.imfs) and np.array_equal(q.residual, r.residual)
    assert q.n_modes == 2 and str(q.stats["method"]) == "gpu" and int(q.stats["E"]) == 4
    assert M.EMDResult(imfs=r.imfs, residual=r.residual, n_modes=2).recon_error() == 0.0


def test_reference_noise_streams_equal_oracle():
    x = np.sin(np.arange(300) * 0.1)
    a = M.reference_noise(x, 5, 0.2, 7, "reference-gpu")
    b = O.noise_gpu_stream(x, 5, 0.2, 7)
    assert np.array_equal(a, b)
    a = M.reference_noise(x, 5, 0.2, 7, "reference-cpu")
    b = O.noise_cpu_stream(x, 5, 0.2, 7)
    assert np.array_equal(a, b)


def test_imf_slots():
    assert M.imf_slots(1000, 5) == 5
    assert M.imf_slots(48000, -1) == 24
    assert M.imf_slots(8, -1) == 11
    assert M.imf_slots(1 << 40, -1) == 48
    with pytest.raises(ValueError):
        M.imf_slots(100, 0)


def test_make_params_validation():
    with pytest.raises(ValueError):
        M.make_params(end="periodic")
    with pytest.raises(ValueError):
        M.make_params(rules="matlab")
    with pytest.raises(ValueError):
        M.make_params(dtype=np.float16)
    with pytest.raises(ValueError):
        M.make_params(dtype=np.float32, exact=True)
    p = M.make_params(dtype=np.float32, end="mirror", rules="numba", max_sifts=10, max_imf=8)
    assert p.dtype == 1 and p.end_mode == 1 and p.rules == 1 and p.max_sifts == 10


def test_decompose_many_validates_before_the_device():
    from eemd4cuda_b200 import emd_par as M
    assert M.decompose_many([]) == []
    with pytest.raises(ValueError):
        M.decompose_many([np.ones(100), np.ones(5)])
    with pytest.raises(ValueError):
        M.decompose_many([np.ones((2, 50))])
    with pytest.raises(ValueError):
        M.decompose_many([np.ones(100)], E=0)
