"""Trial-sharded ensembles: the partition, the ordered reduction, and two
gloo ranks on CPU.

The engine itself needs a GPU, so the CPU tests give decompose_sharded a
runner that computes one trial block with the CPU oracle (x plus a per-trial
noise draw, emd_1d per trial, per-mode sums in trial order -- the order the
device reduction uses).  Two ranks must reproduce, bit for bit, one process
that computes the same two blocks and adds them in order.
"""
import os
import socket

import numpy as np
import pytest

from eemd4cuda_b200 import sharded as SH
from oracle import emd_oracle as O

torch = pytest.importorskip("torch")


def oracle_block(x, b0, b1, *, eps, tau, max_sifts, max_imf, min_extrema, end, seed, rules, dtype,
                 config):
    """Per-mode sums and counts of trials b0..b1-1 with the CPU oracle."""
    N = len(x)
    s = np.zeros((max_imf, N))
    c = np.zeros((max_imf,), dtype=np.int32)
    acc = [None] * max_imf
    sigma = eps * np.std(x)
    for e in range(b0, b1):
        noise = np.random.default_rng(seed * 100003 + e).standard_normal(N) * sigma
        imfs, _, _ = O.emd_1d(x + noise, tau=tau, max_sifts=max_sifts, max_imf=max_imf,
                              min_extrema=min_extrema, end=end)
        for m in range(min(len(imfs), max_imf)):
            acc[m] = imfs[m].copy() if acc[m] is None else acc[m] + imfs[m]
            c[m] += 1
    for m in range(max_imf):
        if acc[m] is not None:
            s[m] = s[m] + acc[m]
    return s, c


def _signal(N=600):
    t = np.arange(N)
    return np.sin(0.07 * t) + 0.4 * np.sin(0.31 * t + 0.2) + 0.05 * np.cos(1.3 * t)


KW = dict(E=5, eps=0.2, tau=0.25, max_sifts=8, max_imf=5, seed=3)


def test_trial_blocks_cover_the_ensemble():
    for E in (1, 5, 64, 100, 257):
        for W in (1, 2, 3, 8):
            bl = SH.trial_blocks(E, W)
            assert bl[0][0] == 0 and bl[-1][1] == E
            assert all(a[1] == b[0] for a, b in zip(bl, bl[1:]))
            sizes = [b - a for a, b in bl]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        SH.trial_blocks(0, 2)


def test_single_process_sharded_equals_oracle_ensemble():
    x = _signal()
    r = SH.decompose_sharded(x, runner=oracle_block, **KW)
    s, c = oracle_block(x, 0, KW["E"], eps=0.2, tau=0.25, max_sifts=8, max_imf=5, min_extrema=4,
                        end="natural", seed=3, rules="ref", dtype=np.float64, config=None)
    means, resid, nm = SH.finalize_host(x, s, c)
    assert r.n_modes == nm
    assert np.array_equal(r.imfs, means) and np.array_equal(r.residual, resid)
    assert r.recon_error() <= 1e-12 * np.abs(x).max()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r = SH.decompose_sharded(_signal(), runner=oracle_block, **KW)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), imfs=r.imfs, residual=r.residual,
                 n_modes=r.n_modes, world=r.stats["world"])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_the_same_blocks_in_one_process(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    a = np.load(tmp_path / "rank0.npz")
    b = np.load(tmp_path / "rank1.npz")
    assert int(a["world"]) == world
    assert np.array_equal(a["imfs"], b["imfs"]) and np.array_equal(a["residual"], b["residual"])
    # one process: the same two blocks, added in rank order
    x = _signal()
    kw = dict(eps=0.2, tau=0.25, max_sifts=8, max_imf=5, min_extrema=4, end="natural", seed=3,
              rules="ref", dtype=np.float64, config=None)
    blocks = SH.trial_blocks(KW["E"], world)
    parts = [oracle_block(x, b0, b1, **kw) for b0, b1 in blocks]
    total, count = SH.combine_blocks([p[0] for p in parts], [p[1] for p in parts])
    means, resid, nm = SH.finalize_host(x, total, count)
    assert int(a["n_modes"]) == nm
    assert np.array_equal(a["imfs"], means) and np.array_equal(a["residual"], resid)
    # and agrees with the unsharded ensemble up to summation grouping
    s, c = oracle_block(x, 0, KW["E"], **kw)
    m1, r1, _ = SH.finalize_host(x, s, c)
    assert np.allclose(a["imfs"], m1, rtol=0, atol=1e-12 * np.abs(x).max())


@pytest.mark.gpu
def test_sharded_single_process_equals_decompose_on_the_gpu():
    """One process, one block: the same sums the batched engine forms."""
    from eemd4cuda_b200 import emd_par as M
    from eemd4cuda_b200 import signals
    x = signals.harmonic_clicks(6000, seed=2)
    a = SH.decompose_sharded(x, E=6, eps=0.2, tau=0.25, max_sifts=20, max_imf=6, seed=4)
    b = M.decompose(x, E=6, eps=0.2, tau=0.25, max_sifts=20, max_imf=6, seed=4, batch=6)
    assert a.n_modes == b.n_modes
    assert np.array_equal(a.imfs, b.imfs)
    assert np.array_equal(a.residual, b.residual)
