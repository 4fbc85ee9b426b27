"""Batch-granularity checkpoint of an ensemble run: the file logic (CPU) and
an interrupted run resumed on the device (GPU).  The interruption is made on
the host: the engine call raises after two batches."""
import numpy as np
import pytest

from eemd4cuda_b200 import _lib as L
from eemd4cuda_b200 import emd_par as M


def _key(x, **over):
    kw = dict(E=8, eps=0.2, tau=0.25, max_sifts=50, max_imf=10, min_extrema=4, end="natural",
              seed=3, noise="philox", rules="ref", exact=False, dtype=np.float64, config=None)
    kw.update(over)
    return M.checkpoint_key(x, **kw)


def test_checkpoint_round_trip_and_refusal(tmp_path):
    x = np.sin(np.arange(1000) * 0.1)
    path = tmp_path / "run.npz"
    ck = M.Checkpoint(path, _key(x))
    assert ck.load() is None
    s = np.arange(20, dtype=np.float64).reshape(2, 10)
    ck.save(batch=4, next_trial=4, imf_sum=s, mode_count=np.array([4, 3], np.int32),
            counters=np.ones((3, 4), np.int32))
    st = M.Checkpoint(path, _key(x)).load()
    assert int(st["batch"]) == 4 and int(st["next"]) == 4
    assert np.array_equal(st["imf_sum"], s) and st["counters"].shape == (3, 4)
    # another signal, seed or engine setting is a different run
    for other in (_key(x + 1e-12), _key(x, seed=4), _key(x, config=M.EngineConfig(halo=20))):
        with pytest.raises(ValueError):
            M.Checkpoint(path, other).load()
    ck.remove()
    assert not path.exists()


@pytest.mark.gpu
def test_interrupted_run_resumes_bit_identical(tmp_path, monkeypatch):
    from eemd4cuda_b200 import signals
    x = signals.harmonic_clicks(48000, seed=1)
    kw = dict(E=20, eps=0.2, tau=0.0, max_sifts=10, max_imf=8, seed=5, batch=5)
    whole = M.decompose(x, **kw)

    path = tmp_path / "eemd.npz"
    real_run = L.run
    calls = {"n": 0}

    def failing_run(*a, **k):
        if calls["n"] == 2:
            raise RuntimeError("simulated interruption")
        calls["n"] += 1
        return real_run(*a, **k)

    monkeypatch.setattr(L, "run", failing_run)
    with pytest.raises(RuntimeError, match="simulated"):
        M.decompose(x, checkpoint=path, **kw)
    monkeypatch.setattr(L, "run", real_run)
    st = M.Checkpoint(path, M.checkpoint_key(
        x, E=20, eps=0.2, tau=0.0, max_sifts=10, max_imf=M.imf_slots(len(x), 8), min_extrema=4,
        end="natural", seed=5, noise="philox", rules="ref", exact=False, dtype=np.float64,
        config=None)).load()
    assert int(st["next"]) == 10  # two batches of 5 trials were saved

    with pytest.raises(ValueError):
        M.decompose(x, checkpoint=path, **dict(kw, batch=4))  # other batch boundaries
    resumed = M.decompose(x, checkpoint=path, **kw)
    assert not path.exists()
    assert resumed.n_modes == whole.n_modes
    assert np.array_equal(resumed.imfs, whole.imfs)
    assert np.array_equal(resumed.residual, whole.residual)
    assert np.array_equal(resumed.stats["per_trial_total_sifts"], whole.stats["per_trial_total_sifts"])
    assert np.array_equal(resumed.stats["per_trial_n_modes"], whole.stats["per_trial_n_modes"])
