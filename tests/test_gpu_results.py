"""Result files written from device tensors, asynchronously, equal the ones
written from host arrays."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from eemd4cuda_b200 import results  # noqa: E402


def test_async_writer_files_equal_host_written_files(tmp_path):
    rng = np.random.default_rng(1)
    N, K = 48000, 8
    segs = []
    for s in range(3):
        x = rng.standard_normal(N)
        imfs = rng.standard_normal((K, N))
        segs.append((x, np.arange(N) / 48000.0, imfs, x - imfs.sum(axis=0),
                     dict(E=100, total_sifts=800 + s, per_mode_sifts=[10] * K)))
    w = results.AsyncWriter()
    for s, (x, t, imfs, res, st) in enumerate(segs):
        d = tmp_path / f"dev{s}"
        d.mkdir()
        # device tensors produced on the current stream, then overwritten only after wait_copies
        im_d = torch.from_numpy(imfs).cuda() * 1.0
        r_d = torch.from_numpy(res).cuda() * 1.0
        w.submit(d, x, t, im_d, r_d, K, st)
    w.close()
    for s, (x, t, imfs, res, st) in enumerate(segs):
        h = tmp_path / f"host{s}"
        h.mkdir()
        results.write_imfs_npz(h, x, t, imfs, res, K, st)
        a, b = np.load(tmp_path / f"dev{s}" / "imfs.npz"), np.load(h / "imfs.npz")
        assert sorted(a.files) == sorted(b.files)
        for k in a.files:
            assert np.array_equal(a[k], b[k]), (s, k)
    # EMDResult's file from device tensors
    x, t, imfs, res, st = segs[0]
    results.save_result(tmp_path / "r.npz", torch.from_numpy(imfs).cuda(), torch.from_numpy(res).cuda(), K, st)
    d = np.load(tmp_path / "r.npz")
    assert np.array_equal(d["imfs"], imfs) and int(d["n_modes"]) == K


def test_pipelined_segments_equal_one_decomposition_per_segment(tmp_path):
    from eemd4cuda_b200 import audio, signals
    from eemd4cuda_b200 import emd_par as M
    sr = 8000
    x = signals.harmonic_clicks(20500, seed=3, fs=float(sr))
    kw = dict(E=16, eps=0.2, tau=0.25, max_sifts=20, max_imf=6)
    segs = audio.decompose_segments(x, sr, segment_s=1.0, seed=7, outdir=tmp_path, **kw)
    assert len(segs) == 3  # 8000, 8000, 4500 samples
    bounds = [(0, 8000), (8000, 16000), (16000, 20500)]
    for k, ((a, b), (imfs, res)) in enumerate(zip(bounds, segs)):
        r = M.decompose(x[a:b].astype(np.float32), seed=7 + k, dtype=np.float32, **kw)
        assert r.n_modes == imfs.shape[0]
        assert np.array_equal(r.imfs, imfs) and np.array_equal(r.residual, res)
        d = np.load(tmp_path / f"seg_{k:04d}" / "imfs.npz")
        assert np.array_equal(d["imfs"], imfs) and int(d["n_modes"]) == imfs.shape[0]
