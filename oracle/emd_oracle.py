"""CPU oracle for the EEMD hot path -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy, the reference algorithm of
misureaudio/EEMD4CUDA so the GPU engine can be checked against it.  It is
imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg; the product (eemd4cuda_b200) never calls it.

Pinned against the reference: tests/golden/ holds fixtures produced by the
reference's own emd_ref.py (and its numba kernel run under numba's CUDA
simulator) by tests/golden/make_golden.py; tests/test_oracle_golden.py checks
this restatement against them (integers exactly, floats to 1e-12).

Followed reference lines (misureaudio/EEMD4CUDA):
  emd_ref.py:31-48   _build_interior_system / _rhs  -> spline_system()
  emd_ref.py:50-65   thomas                          -> thomas()
  emd_ref.py:67-75   _spline_eval                    -> spline_eval()
  emd_ref.py:77-103  envelope (natural / mirror)     -> envelope()
  emd_ref.py:108-156 emd_1d                          -> emd_1d()
  emd_gpu.py:152-274 numba kernel stop rules         -> emd_1d(rules='numba')
  emd_par.py:117-118, 225-233  noise streams         -> noise_*()
  emd_par.py:123-137, 241-250  ensemble mean         -> ensemble_mean()
  emd_gpu_v5_dsbt.py:51-74 + audit_eemd/test_block_thomas.py:86-114
                     seam-window Thomas (owned-only) -> dsbt_solve()
  audit_eemd/test_block_thomas.py:121-133 tile scan  -> scan_tiles()
  emd_ref.py:158-162, 166-168, 220-259 CEEMDAN        -> ceemdan()
"""
from __future__ import annotations

import math
import time

import numpy as np

# ---------------------------------------------------------------------------
# extrema
# ---------------------------------------------------------------------------


def extrema(x: np.ndarray):
    """Indices of strict interior maxima and minima (emd_ref.py:84-87)."""
    c = x[1:-1]
    imax = np.flatnonzero((c > x[:-2]) & (c > x[2:])) + 1
    imin = np.flatnonzero((c < x[:-2]) & (c < x[2:])) + 1
    return imax, imin


def scan_tiles(x: np.ndarray, want_max: bool, tile: int = 128) -> np.ndarray:
    """Tile-ordered compaction of strict extrema, the device's scan order
    (audit_eemd/test_block_thomas.py:121-133): per tile of `tile` samples the
    hits are compacted in time order behind the running total of the earlier
    tiles.  Must equal the serial scan."""
    n = len(x)
    if n < 3:
        return np.zeros(0, dtype=np.int64)
    c = x[1:-1]
    hits = ((c > x[:-2]) & (c > x[2:])) if want_max else ((c < x[:-2]) & (c < x[2:]))
    out = []
    for base in range(1, n - 1, tile):
        stop = min(base + tile, n - 1)
        sel = np.flatnonzero(hits[base - 1:stop - 1])
        out.extend((base + sel).tolist())
    return np.asarray(out, dtype=np.int64)


# ---------------------------------------------------------------------------
# spline system and solves
# ---------------------------------------------------------------------------


def spline_system(tm: np.ndarray, ym: np.ndarray):
    """Interior system of the natural cubic spline through (tm, ym)
    (emd_ref.py:31-48): rows q=0..n-1 for M[q+1], n = p-2,
      d = 2(H_q + H_{q+1}), l = H_q (q>=1), u = H_{q+1} (q<=n-2),
      r = 6((y_{q+2}-y_{q+1})/H_{q+1} - (y_{q+1}-y_q)/H_q)."""
    H = np.diff(tm)
    n = len(tm) - 2
    dg = 2.0 * (H[:n] + H[1:n + 1])
    lo = np.zeros(n)
    up = np.zeros(n)
    lo[1:] = H[1:n]
    up[:n - 1] = H[1:n]
    r = 6.0 * ((ym[2:n + 2] - ym[1:n + 1]) / H[1:n + 1] - (ym[1:n + 1] - ym[:n]) / H[:n])
    return dg, lo, up, r


def thomas(dg, lo, up, r) -> np.ndarray:
    """Serial no-pivot Thomas (emd_ref.py:50-65), same operation order."""
    n = len(dg)
    if n == 0:
        return np.zeros(0)
    dg = dg.tolist(); lo = lo.tolist(); up = up.tolist(); r = r.tolist()
    cs = [0.0] * n
    ds = [0.0] * n
    cs[0] = (up[0] if n > 1 else 0.0) / dg[0]
    ds[0] = r[0] / dg[0]
    for i in range(1, n):
        den = dg[i] - lo[i] * cs[i - 1]
        cs[i] = (up[i] if i < n - 1 else 0.0) / den
        ds[i] = (r[i] - lo[i] * ds[i - 1]) / den
    xs = [0.0] * n
    xs[-1] = ds[-1]
    for i in range(n - 2, -1, -1):
        xs[i] = ds[i] - cs[i] * xs[i + 1]
    return np.asarray(xs)


def window_thomas(dg, lo, up, r, w0: int, w1: int) -> np.ndarray:
    """Thomas on rows [w0, w1] with the couplings outside the window dropped
    (emd_gpu_v5_dsbt.py:51-74).  Returns the window solution."""
    m = w1 - w0 + 1
    cs = [0.0] * m
    ds = [0.0] * m
    cp = 0.0
    dp = 0.0
    for k in range(m):
        i = w0 + k
        den = dg[i] - lo[i] * cp
        c = 0.0 if i == w1 else up[i] / den
        dv = (r[i] - lo[i] * dp) / den
        cs[k] = c
        ds[k] = dv
        cp, dp = c, dv
    xs = [0.0] * m
    xs[-1] = ds[-1]
    for k in range(m - 2, -1, -1):
        xs[k] = ds[k] - cs[k] * xs[k + 1]
    return np.asarray(xs)


def dsbt_solve(dg, lo, up, r, B: int = 250, S: int = 30) -> np.ndarray:
    """Decay-seamed block Thomas: owned blocks of B rows, each solved on its
    window [o0-S, o1+S] (clipped); only the owned rows are kept
    (audit_eemd/test_block_thomas.py:86-114, the fixed owned-only mirror)."""
    n = len(dg)
    x = np.zeros(n)
    dg = np.asarray(dg).tolist(); lo = np.asarray(lo).tolist()
    up = np.asarray(up).tolist(); r = np.asarray(r).tolist()
    for o0 in range(0, n, B):
        o1 = min(n, o0 + B) - 1
        w0 = max(0, o0 - S)
        w1 = min(n - 1, o1 + S)
        xw = window_thomas(dg, lo, up, r, w0, w1)
        x[o0:o1 + 1] = xw[o0 - w0:o1 - w0 + 1]
    return x


def spline_eval(tm, ym, M, t) -> np.ndarray:
    """Cubic spline with second derivatives M at points t (emd_ref.py:67-75):
    interval = searchsorted-left minus one, clipped to [0, p-2]."""
    p = len(tm)
    idx = np.clip(np.searchsorted(tm, t) - 1, 0, p - 2)
    t1 = tm[idx + 1]
    t0 = tm[idx]
    h = t1 - t0
    a = (t1 - t) / h
    b = (t - t0) / h
    return (a * ym[idx] + b * ym[idx + 1]
            + ((a ** 3 - a) * M[idx] + (b ** 3 - b) * M[idx + 1]) * (h * h) / 6.0)


def envelope(t, x, kind: str, end: str = "natural", solver=None):
    """Spline envelope through the strict maxima ('max') or minima ('min')
    evaluated at t (emd_ref.py:77-103).  Returns (env, n_knots)."""
    imax, imin = extrema(x)
    k = imax if kind == "max" else imin
    p = len(k)
    if p < 2:
        return np.full_like(t, x[k[0]] if p == 1 else 0.0), p
    tm = t[k]
    ym = x[k]
    if end == "mirror" and p >= 3:
        tm = np.concatenate(([tm[0] - (tm[1] - tm[0])], tm, [tm[-1] + (tm[-1] - tm[-2])]))
        ym = np.concatenate(([ym[1]], ym, [ym[-2]]))
    dg, lo, up, r = spline_system(tm, ym)
    Mi = (solver or thomas)(dg, lo, up, r)
    M = np.zeros(len(tm))
    M[1:-1] = Mi
    return spline_eval(tm, ym, M, t), p


# ---------------------------------------------------------------------------
# EMD
# ---------------------------------------------------------------------------


def emd_1d(x, tau=0.25, max_sifts=50, max_imf=-1, min_extrema=4, end="natural",
           rules="ref", solver=None, record_knots=False):
    """Full EMD of one signal (emd_ref.py:108-156).

    rules='ref'   emd_ref stop rules: IMF loop ends when nmax+nmin < min_extrema
                  or max_imf reached; a sift is skipped (IMF closes) when
                  nmax<1 or nmin<1; SD = sum((h-h_new)^2)/sum(h^2) from the 2nd sift.
    rules='numba' emd_gpu.py:152-274: the IMF loop also ends when nmax<2 or
                  nmin<2, a sift is skipped when nmax<2 or nmin<2, SD = sum(m^2)/sum(h^2).
    Returns (imfs list, residual, stats) with stats n_modes, total_sifts,
    per_mode_sifts and (record_knots) knot_log[m][k] = (nmax, nmin)."""
    x = np.asarray(x, dtype=float)
    t = np.arange(len(x), dtype=float)
    numba = rules == "numba"
    imfs = []
    resid = x.copy()
    total = 0
    per_mode = []
    klog = []
    while True:
        imax, imin = extrema(resid)
        nmax, nmin = len(imax), len(imin)
        if nmax + nmin < min_extrema:
            break
        if numba and (nmax < 2 or nmin < 2):
            break
        if max_imf != -1 and len(imfs) >= max_imf:
            break
        h = resid.copy()
        ns = 0
        mlog = []
        for k in range(max_sifts):
            imax, imin = extrema(h)
            if numba:
                if len(imax) < 2 or len(imin) < 2:
                    break
            elif len(imax) < 1 or len(imin) < 1:
                break
            mlog.append((len(imax), len(imin)))
            eu, _ = envelope(t, h, "max", end, solver)
            el, _ = envelope(t, h, "min", end, solver)
            m = 0.5 * (eu + el)
            h_new = h - m
            ns += 1
            if k >= 1:
                num = np.sum(m ** 2) if numba else np.sum((h - h_new) ** 2)
                den = np.sum(h ** 2)
                sd = num / den if den > 0 else 0.0
                if sd < tau:
                    h = h_new
                    break
            h = h_new
        imfs.append(h)
        per_mode.append(ns)
        klog.append(mlog)
        total += ns
        resid = resid - h
    stats = dict(n_modes=len(imfs), total_sifts=total, per_mode_sifts=per_mode)
    if record_knots:
        stats["knot_log"] = klog
    return imfs, resid, stats


def one_sift(x, end="natural"):
    """h - mean envelope for one sift of x (test_emd_gpu.py:89-102 A1)."""
    t = np.arange(len(x), dtype=float)
    eu, _ = envelope(t, x, "max", end)
    el, _ = envelope(t, x, "min", end)
    return x - 0.5 * (eu + el)


# ---------------------------------------------------------------------------
# ensemble
# ---------------------------------------------------------------------------


def noise_gpu_stream(x, E, eps, seed):
    """emd_par.py:225,233 -- one default_rng(seed) draw of (E, N) * eps*std(x)."""
    return np.random.default_rng(seed).standard_normal((E, len(x))) * (eps * np.std(x))


def noise_cpu_stream(x, E, eps, seed):
    """emd_par.py:117-118 -- per-trial default_rng((seed*1000003+e) mod 2^64)."""
    sigma = eps * np.std(x)
    out = np.empty((E, len(x)))
    for e in range(E):
        out[e] = np.random.default_rng((seed * 1000003 + e) & 0xFFFFFFFFFFFFFFFF) \
            .standard_normal(len(x)) * sigma
    return out


def ensemble_mean(x, trial_imfs):
    """Per-mode mean over the trials that produced the mode, summed in trial
    order, and residual x - sum(mean) (emd_par.py:241-250)."""
    N = len(x)
    maxm = max((len(t) for t in trial_imfs), default=0)
    avg = np.zeros((maxm, N))
    cnt = np.zeros(maxm)
    for m in range(maxm):
        rows = [np.asarray(t[m]) for t in trial_imfs if len(t) > m]
        if rows:
            avg[m] += np.stack(rows).sum(axis=0)
            cnt[m] += len(rows)
    n_modes = int((cnt > 0).sum())
    avg = avg[:n_modes] / np.where(cnt[:n_modes] > 0, cnt[:n_modes], 1)[:, None]
    return avg, x - avg.sum(axis=0), cnt[:n_modes]


def eemd(x, X, **kw):
    """EEMD of the perturbed trials X [E, N]; returns (mean, residual, per-trial results)."""
    res = [emd_1d(X[e], **kw) for e in range(X.shape[0])]
    avg, resid, _ = ensemble_mean(x, [r[0] for r in res])
    return avg, resid, res


def ceemdan(x, E=100, eps=0.2, seed=0, tau=0.25, max_sifts=50, end="natural"):
    """CEEMDAN as the reference computes it (emd_ref.py:220-259).

    W = default_rng(seed).standard_normal((E, N)) (emd_ref.py:166-168).
    Stage 0: the full EMD of every W[e]; only its mode count is used (the
    stop test below; the normalised noise IMFs are not added anywhere).
    Stage k: while max|r| >= 1e-12 and std(r) >= 1e-10, beta = eps*std(r),
    c_k = (sum over e, in order, of the first IMF of r + beta*W[e]) / E (first
    IMF: emd_1d with max_imf=1, min_extrema=4, emd_ref.py:158-162), r -= c_k;
    stop after stage k when k >= the mode count of every noise EMD.
    Returns (c [n_imfs, N], r, stats with E, n_imfs, noise_modes, stage_sifts)."""
    x = np.asarray(x, dtype=float)
    N = len(x)
    W = np.random.default_rng(seed).standard_normal((E, N))
    noise_modes = [emd_1d(W[e] + np.zeros(N), tau=tau, max_sifts=max_sifts, min_extrema=4, end=end)[2]["n_modes"]
                   for e in range(E)]
    c_imfs = []
    stage_sifts = []
    resid = x.copy()
    while True:
        if np.max(np.abs(resid)) < 1e-12 or np.std(resid) < 1e-10:
            break
        stage = len(c_imfs)
        beta = eps * np.std(resid)
        c = np.zeros(N)
        sifts = []
        for e in range(E):
            imfs, _, st = emd_1d(resid + beta * W[e], tau=tau, max_sifts=max_sifts, max_imf=1, min_extrema=4,
                                 end=end)
            c += imfs[0]
            sifts.append(st["per_mode_sifts"][0])
        c /= E
        c_imfs.append(c)
        stage_sifts.append(sifts)
        resid = resid - c
        if all(stage >= noise_modes[e] for e in range(E)):
            break
    return np.array(c_imfs), resid, dict(E=E, n_imfs=len(c_imfs), noise_modes=noise_modes,
                                         stage_sifts=stage_sifts)


# ---------------------------------------------------------------------------
# CPU baseline (the reference's process-pool EEMD, emd_par.py:139-183)
# ---------------------------------------------------------------------------


def _trial_worker(args):
    x, noise, kw = args
    t0 = time.perf_counter()
    imfs, resid, st = emd_1d(x + noise, **kw)
    return len(imfs), st["total_sifts"], time.perf_counter() - t0


def _imfs_worker(args):
    """emd_1d of one prepared trial input (float64): the IMF stack [n_modes, N]
    and the per-sift knot counts, for accuracy checks against the engine."""
    x, kw = args
    imfs, _, st = emd_1d(np.asarray(x, dtype=np.float64), record_knots=True, **kw)
    return np.array(imfs), st["knot_log"]


def timed_pool_eemd(x, noises, n_workers, **kw):
    """Run emd_1d on x + noises[e] in a spawn process pool with dynamic
    scheduling; returns (wall seconds, per-trial (n_modes, sifts, seconds))."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor, as_completed

    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    out = []
    with ProcessPoolExecutor(max_workers=n_workers, mp_context=ctx) as ex:
        futs = [ex.submit(_trial_worker, (x, noises[e], kw)) for e in range(len(noises))]
        for f in as_completed(futs):
            out.append(f.result())
    return time.perf_counter() - t0, out
