"""Trial-sharded EEMD over the ranks of a torch.distributed group.

The trials of one ensemble are independent tasks, so an ensemble spreads over
GPUs without any exchange on the data path: rank r of W runs the contiguous
trial block [r*E/W, (r+1)*E/W).  The device noise is keyed by the absolute
trial index, so every rank draws exactly the noise a single-process run would.
Each rank produces its block's per-mode sums ([max_imf, N] float64) and
trial counts ([max_imf] int32); one all_gather of those is the only
collective, and every rank then adds the blocks in rank order -- the order in
which a single process adds consecutive trial batches -- and forms the
per-mode mean and the residual x - sum(mean).  A single-process run whose
batches are the same trial blocks gives bit-identical results.

    res = decompose_sharded(x, E=256, eps=0.2, tau=0.0, max_sifts=10, max_imf=8)

`runner` replaces the GPU engine for one trial block (tests use the CPU
oracle to check the partition and the reduction on gloo ranks).
"""
from __future__ import annotations

import numpy as np

from . import emd_par as M

__all__ = ["trial_blocks", "combine_blocks", "finalize_host", "decompose_sharded"]


def trial_blocks(E: int, world: int) -> list[tuple[int, int]]:
    """Contiguous trial blocks of E trials over `world` ranks (sizes differ by at most 1)."""
    if E < 1 or world < 1:
        raise ValueError("E and world must be >= 1")
    return [(r * E // world, (r + 1) * E // world) for r in range(world)]


def combine_blocks(sums: list[np.ndarray], counts: list[np.ndarray]):
    """Per-mode sums and counts of consecutive trial blocks, added in block order."""
    total = np.zeros_like(sums[0])
    for s in sums:
        total = total + s
    count = np.zeros_like(counts[0])
    for c in counts:
        count = count + c
    return total, count


def finalize_host(x: np.ndarray, imf_sum: np.ndarray, count: np.ndarray):
    """Mean of each mode over the trials that reached it, and x - sum(mean)
    (the same order of operations as the device finalisation,
    emd_par.py:241-250)."""
    n_modes = 0
    while n_modes < len(count) and count[n_modes] > 0:
        n_modes += 1
    means = np.empty((n_modes, imf_sum.shape[1]))
    acc = None
    for m in range(n_modes):
        means[m] = imf_sum[m] / float(count[m])
        acc = means[m].copy() if acc is None else acc + means[m]
    resid = np.asarray(x, dtype=np.float64) - (acc if acc is not None else 0.0)
    return means, resid, n_modes


def _gpu_block(x, b0, b1, *, eps, tau, max_sifts, max_imf, min_extrema, end, seed, rules, dtype,
               config):
    """One trial block on the local GPU: per-mode sums and counts (host arrays)."""
    torch = M._torch()
    from . import _lib as L
    dev = torch.device("cuda", torch.cuda.current_device())
    dt = np.dtype(dtype)
    N = len(x)
    p = M.make_params(dtype=dt, noise_mode=L.EEMD_NOISE_PHILOX, eps=eps, seed=seed, tau=tau,
                      max_sifts=max_sifts, max_imf=max_imf, min_extrema=min_extrema, end=end,
                      rules=rules, config=config)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).to(dev)
    imf_sum = torch.zeros((max_imf, N), dtype=torch.float64, device=dev)
    count = torch.zeros((max_imf,), dtype=torch.int32, device=dev)
    if b1 > b0:
        ws = torch.empty((L.workspace_size(p, [N], b1 - b0, False),), dtype=torch.uint8, device=dev)
        L.run(p, xd, [N], b0, b1 - b0, ws, imf_sum=imf_sum, mode_count=count)
    return imf_sum.cpu().numpy(), count.cpu().numpy()


def decompose_sharded(x, E=64, eps=0.2, tau=0.25, max_sifts=50, max_imf=-1, min_extrema=4,
                      end="natural", seed=0, *, rules="ref", dtype=np.float64, config=None,
                      group=None, runner=None) -> M.EMDResult:
    """EEMD of x with the E trials split over the ranks of `group` (the
    default process group when torch.distributed is initialised, otherwise
    one process).  Every rank returns the same EMDResult."""
    x = np.asarray(x, dtype=float)
    if x.ndim != 1:
        raise ValueError("x must be 1-D")
    if len(x) < 8:
        raise ValueError("signal too short for EMD (need >= 8 samples)")
    E = int(E)
    if E < 2:
        raise ValueError("decompose_sharded needs an ensemble (E >= 2); use decompose for E=1")
    slots = M.imf_slots(len(x), max_imf)
    import torch.distributed as dist
    distributed = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if distributed else 1
    rank = dist.get_rank(group) if distributed else 0
    b0, b1 = trial_blocks(E, world)[rank]
    kw = dict(eps=eps, tau=tau, max_sifts=max_sifts, max_imf=slots, min_extrema=min_extrema,
              end=end, seed=seed, rules=rules, dtype=dtype, config=config)
    run = runner if runner is not None else _gpu_block
    s, c = run(x, b0, b1, **kw)
    if distributed:
        import torch
        # NCCL gathers device tensors, gloo host tensors
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        st = torch.from_numpy(np.ascontiguousarray(s)).to(dev)
        ct = torch.from_numpy(np.ascontiguousarray(c)).to(dev)
        s_all = [torch.empty_like(st) for _ in range(world)]
        c_all = [torch.empty_like(ct) for _ in range(world)]
        dist.all_gather(s_all, st, group=group)
        dist.all_gather(c_all, ct, group=group)
        sums = [t.cpu().numpy() for t in s_all]
        counts = [t.cpu().numpy() for t in c_all]
    else:
        sums, counts = [s], [c]
    total, count = combine_blocks(sums, counts)
    means, resid, n_modes = finalize_host(x, total, count)
    stats = dict(method="gpu", backend="b200", E=E, n_modes=n_modes, world=world,
                 trial_blocks=trial_blocks(E, world), x=x)
    return M.EMDResult(imfs=means, residual=resid, n_modes=n_modes, stats=stats)
