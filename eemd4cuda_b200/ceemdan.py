"""CEEMDAN on the B200 engine, with the reference's semantics (emd_ref.py:220-259).

    c_imfs, resid, stats = ceemdan(x, E=100, eps=0.2, seed=0, tau=0.25, max_sifts=50)

The staircase is sequential over modes and parallel over trials.  Each stage
is one engine launch over the E trials of one signal: trial e sifts only the
first IMF (max_imf = 1, min_extrema = 4) of r + beta * W[e], where W is the
reference's standard-normal draw default_rng(seed).standard_normal((E, N))
(emd_ref.py:166-168), resident on the device for the whole run, and the
engine forms beta * W[e] and the sum each rounded as numpy does
(EEMD_NOISE_SCALED).  The engine adds the trials' first IMFs in trial order
and eemd_finalize divides by E and subtracts the mean from r on the device.
Stage 0 is one launch of the full EMD of every W[e] for its mode count, which
ends the staircase (the reference computes and normalises the noise IMFs but
adds only the raw W; this reproduces that).  beta = eps * std(r) and the
stop tests use numpy on the host copy of r, as the reference does, so the
float64 path matches it operation for operation.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from . import emd_par as M

__all__ = ["ceemdan"]


def ceemdan(x, E=100, eps=0.2, parallel=True, n_workers=None, seed=0, *, tau=0.25, max_sifts=50,
            end="natural", exact=False, noise="reference", config=None, **_ignored):
    """CEEMDAN of x; returns (c_imfs [n_imfs, N] float64, residual [N], stats).

    parallel / n_workers are accepted for signature compatibility (the trials
    of a stage run in one launch).  exact=True solves every spline system with
    the exact serial Thomas order (bit-for-bit with the reference's float64
    operations); the default uses the seam-window solve.  noise="reference"
    draws W with numpy's default_rng(seed) as the reference does (on the host,
    about 10 ns per sample: most of the run's time for E = 100, N = 48000);
    noise="philox" draws it on the device (eemd_philox_normals, keyed by seed
    and trial), the same staircase on a different noise stream."""
    torch = M._torch()
    x = np.asarray(x, dtype=float)
    if x.ndim != 1:
        raise ValueError("x must be 1-D")
    N = len(x)
    if N < 8:
        raise ValueError("signal too short for EMD (need >= 8 samples)")
    E = int(E)
    if E < 1:
        raise ValueError("E must be >= 1")
    dev = torch.device("cuda", torch.cuda.current_device())
    if noise == "reference":
        Wd = torch.from_numpy(np.random.default_rng(seed).standard_normal((E, N))).to(dev)
    elif noise == "philox":
        Wd = torch.empty((E, N), dtype=torch.float64, device=dev)
        L.philox_normals(seed, 0, 0, E, N, Wd)
    else:
        raise ValueError("noise must be 'reference' or 'philox'")

    # stage 0: mode count of the full EMD of every noise row
    slots = M.imf_slots(N, -1)
    p0 = M.make_params(dtype=np.float64, noise_mode=L.EEMD_NOISE_PREPERTURBED, tau=tau, max_sifts=max_sifts,
                       max_imf=slots, min_extrema=4, end=end, exact=exact, config=config)
    p1 = M.make_params(dtype=np.float64, noise_mode=L.EEMD_NOISE_SCALED, eps=0.0, tau=tau, max_sifts=max_sifts,
                       max_imf=1, min_extrema=4, end=end, exact=exact, config=config)
    ws_bytes = max(L.workspace_size(p0, [N], E, False), L.workspace_size(p1, [N], E, False))
    ws = torch.empty((ws_bytes,), dtype=torch.uint8, device=dev)
    nmode = torch.zeros((E,), dtype=torch.int32, device=dev)
    L.run(p0, Wd, [N], 0, E, ws, nmode=nmode)
    noise_modes = nmode.cpu().numpy().tolist()
    if max(noise_modes) >= slots:
        raise RuntimeError(f"a noise EMD reached the {slots}-mode cap")

    # per-stage results stay on the device until the staircase ends: the
    # residual is the only copy back per stage (numpy forms beta and the stop
    # tests from it)
    max_st = max(noise_modes) + 1
    imf_sum = torch.empty((N,), dtype=torch.float64, device=dev)
    cnt_buf = torch.zeros((max_st,), dtype=torch.int32, device=dev)
    c_buf = torch.empty((max_st, N), dtype=torch.float64, device=dev)
    sift_buf = torch.empty((max_st, E), dtype=torch.int32, device=dev)
    nm = torch.empty((1,), dtype=torch.int32, device=dev)
    r_d = torch.from_numpy(x.copy()).to(dev)
    r_next = torch.empty_like(r_d)
    h_r = torch.empty((N,), dtype=torch.float64, pin_memory=True)  # each stage's residual, back to the host
    resid = x.copy()
    n_st = 0
    while True:
        if np.max(np.abs(resid)) < 1e-12 or np.std(resid) < 1e-10:
            break
        stage = n_st
        p1.eps = float(eps * np.std(resid))  # beta of this stage
        imf_sum.zero_()
        cnt = cnt_buf[stage:stage + 1]
        L.run(p1, r_d, [N], 0, E, ws, noise=Wd, imf_sum=imf_sum, mode_count=cnt, nsift=sift_buf[stage])
        L.finalize(p1, r_d, [N], imf_sum, cnt, c_buf[stage], r_next, nm)
        h_r.copy_(r_next, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        resid = h_r.numpy().copy()
        n_st += 1
        r_d, r_next = r_next, r_d
        if all(stage >= m for m in noise_modes):
            break
    # the stages' modes and counters through pinned memory, one synchronisation
    h_c = torch.empty((n_st, N), dtype=torch.float64, pin_memory=True)
    h_cnt = torch.empty((n_st,), dtype=torch.int32, pin_memory=True)
    h_sift = torch.empty((n_st, E), dtype=torch.int32, pin_memory=True)
    h_c.copy_(c_buf[:n_st], non_blocking=True)
    h_cnt.copy_(cnt_buf[:n_st], non_blocking=True)
    h_sift.copy_(sift_buf[:n_st], non_blocking=True)
    torch.cuda.current_stream(dev).synchronize()
    counts = h_cnt.numpy()
    for stage, k in enumerate(counts):
        if int(k) != E:
            raise ValueError(f"CEEMDAN stage {stage}: {E - int(k)} of {E} trials have no first IMF "
                             "(fewer than 4 extrema)")
    sifts = h_sift.numpy().tolist()
    c = h_c.numpy() if n_st else np.zeros((0, N))
    return c, resid, dict(E=E, n_imfs=int(n_st), noise_modes=noise_modes, stage_sifts=sifts, method="gpu",
                          backend="b200", exact=bool(exact), noise=noise)
