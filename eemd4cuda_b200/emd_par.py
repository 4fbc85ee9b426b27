"""Drop-in replacement of the reference's public EMD/EEMD module (emd_par.py).

PUBLIC API (same names, arguments and errors as emd_par.py:1-33, 260-301)
    result = decompose(x, method='auto', E=64, eps=0.2, tau=0.25,
                       max_sifts=50, max_imf=-1, min_extrema=4,
                       end='natural', n_workers=None, seed=0, batch=None)
    result.imfs / .residual / .n_modes / .stats / .recon_error()
    result.save(path) / EMDResult.load(path)
    gpu_eemd_full(X[E,N], E, tau, max_sifts, max_imf) -> (imfs, nsift, nmode)
    make_reference_sweep(...)

Every decomposition runs on the sm_100a engine (libeemd_b200.so); there is
no CPU backend, so method='cpu' raises ValueError.  PyTorch tensors serve as
device buffers only.

Keyword-only extensions:
    noise  'philox' (default): counter-based device noise keyed by
           (seed, trial); 'reference-gpu': the host stream of the reference's
           GPU path (one default_rng(seed) draw of (E, N), emd_par.py:225-233);
           'reference-cpu': the per-trial seeds of its CPU path
           (emd_par.py:117-118).  The two reference streams are drawn on the
           host with numpy and injected, so results match the reference's
           inputs bit for bit.
    rules  'ref' (emd_ref.py stop rules, default) or 'numba' (emd_gpu.py).
    exact  True: reference float64 operation order (parity mode).
    dtype  np.float64 (default) or np.float32 storage.
    checkpoint  path of a .npz that an ensemble (E > 1) run updates after
           every trial batch (device sums, mode counts, per-trial counters,
           next trial); a later call with the same arguments and signal
           resumes from it, with results bit-identical to an uninterrupted
           run, and the file is removed once the run completes.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import threading
import time
from dataclasses import asdict, dataclass, field

import numpy as np

from . import _lib as L
from .hostcopy import copy_into, fresh_copy, prefault

__all__ = ["decompose", "decompose_many", "EMDResult", "make_reference_sweep", "gpu_eemd_full", "EngineConfig"]


# =====================================================================
# Result container (emd_par.py:67-97)
# =====================================================================
@dataclass
class EMDResult:
    imfs: np.ndarray          # [n_modes, N]
    residual: np.ndarray      # [N]
    n_modes: int
    stats: dict = field(default_factory=dict)

    def recon_error(self) -> float:
        """Partition-of-unity check: max|x - (sum(imfs)+residual)| (0 if x not stored)."""
        recon = self.imfs.sum(axis=0) + self.residual
        x = self.stats.get("x", None)
        if x is None:
            return 0.0
        return float(np.max(np.abs(x - recon)))

    def save(self, path: str):
        scalars = {k: v for k, v in self.stats.items()
                   if isinstance(v, (int, float, str, np.integer, np.floating))
                   and k not in ("n_modes",)}
        np.savez_compressed(path, imfs=self.imfs, residual=self.residual,
                            n_modes=self.n_modes, **scalars)

    @staticmethod
    def load(path: str) -> "EMDResult":
        d = np.load(path, allow_pickle=False)
        return EMDResult(imfs=d["imfs"], residual=d["residual"], n_modes=int(d["n_modes"]),
                         stats={k: d[k] for k in d.files
                                if k not in ("imfs", "residual", "n_modes")})


@dataclass
class EngineConfig:
    """Engine knobs beyond the reference's signature (0 = default / autotune).

    tile: samples per warp tile; only 32 x 8 (float32) or 32 x 4 (float64).
    knots_per_block: owned rows of an exact-mode seam window; halo: the decay
        halo of every seam window (exact and fast).
    watchdog: negative -k is the test mode (each task first polls a flag that
        nothing sets k times, then the run fails with EEMD_E_TIMEOUT); 0 or
        positive has no effect.
    cluster_size: CTAs sharing one signal (1..16; 9..16 are non-portable cluster sizes).
    cta_warps: warps per CTA (4 or 5; 0 = the autotune table's choice, else 4)."""
    tile: int = 0
    knots_per_block: int = 0
    halo: int = 0
    watchdog: int = 0
    cluster_size: int = 0
    cta_warps: int = 0


_RULES = {"ref": L.EEMD_RULES_REF, "numba": L.EEMD_RULES_NUMBA}
_ENDS = {"natural": L.EEMD_END_NATURAL, "mirror": L.EEMD_END_MIRROR}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the B200 EEMD engine needs a CUDA device (no CPU fallback)")
    return torch


def imf_slots(N: int, max_imf: int) -> int:
    """IMF slots per trial: max_imf, or for max_imf=-1 a bound on the number of
    modes of an N-sample signal (each IMF removes the fastest oscillation; the
    reference's GPU path caps at 64, emd_par.py:205-206)."""
    if max_imf is not None and max_imf != -1:
        if max_imf < 1:
            raise ValueError("max_imf must be -1 or >= 1")
        return int(max_imf)
    return int(min(64, max(8, math.ceil(math.log2(max(N, 2))) + 8)))


def make_params(*, dtype=np.float64, noise_mode=L.EEMD_NOISE_NONE, eps=0.2, seed=0, tau=0.25,
                max_sifts=50, max_imf=16, min_extrema=4, end="natural", rules="ref",
                exact=False, config: EngineConfig | None = None) -> L.EemdParams:
    if end not in _ENDS:
        raise ValueError("end must be 'natural' or 'mirror'")
    if rules not in _RULES:
        raise ValueError("rules must be 'ref' or 'numba'")
    if int(max_sifts) < 1:
        raise ValueError("max_sifts must be >= 1")
    dt = np.dtype(dtype)
    if dt not in (np.dtype(np.float64), np.dtype(np.float32)):
        raise ValueError("dtype must be float64 or float32")
    if exact and dt != np.dtype(np.float64):
        raise ValueError("exact mode needs float64")
    cfg = config or EngineConfig()
    p = L.default_params()
    p.dtype = L.EEMD_F64 if dt == np.dtype(np.float64) else L.EEMD_F32
    p.noise_mode = int(noise_mode)
    p.eps = float(eps)
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    p.tau = float(tau)
    p.max_sifts = int(max_sifts)
    p.max_imf = int(max_imf)
    p.min_extrema = int(min_extrema)
    p.end_mode = _ENDS[end]
    p.rules = _RULES[rules]
    p.exact = 1 if exact else 0
    p.tile = int(cfg.tile)
    p.knots_per_block = int(cfg.knots_per_block)
    p.halo = int(cfg.halo)
    p.watchdog = int(cfg.watchdog)
    p.cluster_size = int(cfg.cluster_size)
    p.cta_warps = int(cfg.cta_warps)
    return p


def tuned(p: L.EemdParams, lengths, trial_count: int) -> L.EemdParams:
    """The parameters of one launch with the threads per trial (CTAs per task
    and warps per CTA) from the autotune table (eemd4cuda_b200/tuning/) when
    the caller left cluster_size and cta_warps at 0; otherwise, or without a
    table entry, p unchanged (the engine then applies its own rule)."""
    from . import autotune

    if p.cluster_size or p.cta_warps:
        return p
    ls = sorted(int(n) for n in lengths)
    # an uneven batch is looked up by its median length (most of its work),
    # with the shortest signal bounding the CTAs per task
    c, nw = autotune.launch_shape(ls[len(ls) // 2], len(ls) * int(trial_count),
                                  "f32" if p.dtype == L.EEMD_F32 else "f64", n_min=ls[0])
    if not c:
        return p
    q = L.EemdParams.from_buffer_copy(p)
    q.cluster_size = c
    q.cta_warps = nw if (nw and not p.exact) else 0
    return q


def _tdtype(torch, dt):
    return torch.float64 if np.dtype(dt) == np.dtype(np.float64) else torch.float32


def reference_noise(x: np.ndarray, E: int, eps: float, seed: int, stream: str) -> np.ndarray:
    """The reference's own noise arrays, scaled by eps*std(x).
    'reference-gpu': emd_par.py:225,233 (one default_rng(seed) stream, (E, N));
    'reference-cpu': emd_par.py:117-118 (default_rng((seed*1000003+e) mod 2^64) per trial)."""
    N = len(x)
    sigma = eps * np.std(x)
    if stream == "reference-gpu":
        return np.random.default_rng(seed).standard_normal((E, N)) * sigma
    if stream == "reference-cpu":
        out = np.empty((E, N))
        for e in range(E):
            rng = np.random.default_rng((seed * 1000003 + e) & 0xFFFFFFFFFFFFFFFF)
            out[e] = rng.standard_normal(N) * sigma
        return out
    raise ValueError("unknown noise stream %r" % (stream,))


_TOTAL_MEM = {}


def _auto_batch(torch, p, N, E, bytes_per_el):
    """Trials resident at once: 70 % of free device memory (emd_par.py:214-223).
    The free-memory query (a driver round trip) is skipped when the whole
    ensemble's workspace is under a tenth of the device's memory."""
    per_trial = L.workspace_size(p, [N], 1, False)
    dev = torch.cuda.current_device()
    if dev not in _TOTAL_MEM:
        _TOTAL_MEM[dev] = torch.cuda.get_device_properties(dev).total_memory
    if per_trial * E < _TOTAL_MEM[dev] // 10:
        return E
    free, _ = torch.cuda.mem_get_info()
    b = max(1, int(free * 0.7 // max(per_trial, 1)))
    return min(E, b)


_STAGE = {}
_STAGE_LOCK = threading.Lock()


# results up to this size come back in pinned host tensors of their own from
# torch's caching host allocator: the device-to-host copies land in memory
# that is already paged in, and the returned arrays are views of it (they keep
# the tensor, and so the block, alive); larger results go through the shared
# staging buffers into fresh arrays
PINNED_RESULT_BYTES = 64 << 20


def _pinned(torch, shape, dtype):
    return torch.empty(shape, dtype=dtype, pin_memory=True)


def _staging(torch, slots, N):
    """Pinned host buffers for the outputs of one shape (the latest shape only is kept)."""
    key = (slots, N)
    if key not in _STAGE:
        _STAGE.clear()
        _STAGE[key] = (torch.empty((slots, N), dtype=torch.float64, pin_memory=True),
                       torch.empty((N,), dtype=torch.float64, pin_memory=True),
                       torch.empty((1,), dtype=torch.int32, pin_memory=True))
    return _STAGE[key]


class Checkpoint:
    """Batch-granularity state of one ensemble run in a .npz file.

    `key` identifies the run (every argument that changes the result, and a
    SHA-256 of the signal); a file written by a different run is refused
    rather than mixed in.  Writes go to a temporary file that replaces the
    old one, so an interruption leaves the previous complete state."""

    def __init__(self, path, key: dict):
        self.path = os.fspath(path)
        self.key = json.dumps(key, sort_keys=True)

    def load(self):
        """The saved state (dict) or None when there is no file."""
        if not os.path.exists(self.path):
            return None
        with np.load(self.path, allow_pickle=False) as z:
            if str(z["key"]) != self.key:
                raise ValueError(f"checkpoint {self.path} was written by a different run "
                                 "(other arguments or signal)")
            return {k: z[k] for k in ("batch", "next", "imf_sum", "mode_count", "counters")}

    def save(self, *, batch, next_trial, imf_sum, mode_count, counters):
        tmp = self.path + ".tmp"
        with open(tmp, "wb") as f:
            np.savez(f, key=np.array(self.key), batch=np.int64(batch), next=np.int64(next_trial),
                     imf_sum=imf_sum, mode_count=mode_count, counters=counters)
        os.replace(tmp, self.path)

    def remove(self):
        if os.path.exists(self.path):
            os.remove(self.path)


def checkpoint_key(x, **kw) -> dict:
    """Identity of an ensemble run for Checkpoint: the arguments and the signal's hash."""
    cfg = kw.pop("config", None)
    kw["config"] = asdict(cfg) if cfg is not None else None
    kw["dtype"] = np.dtype(kw["dtype"]).str
    kw["x_sha256"] = hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()
    kw["N"] = int(len(x))
    return kw


def _run_ensemble(x, *, E, eps, tau, max_sifts, max_imf, min_extrema, end, seed, batch,
                  noise, rules, exact, dtype, config, checkpoint=None):
    """EEMD of one signal: batches of trials into device sums, then mean/residual."""
    torch = _torch()
    nvtx = torch.cuda.nvtx
    N = len(x)
    slots = imf_slots(N, max_imf)
    dt = np.dtype(dtype)
    tdt = _tdtype(torch, dt)
    dev = torch.device("cuda", torch.cuda.current_device())
    if E == 1:
        nmode_kind = L.EEMD_NOISE_NONE
    elif noise == "philox":
        nmode_kind = L.EEMD_NOISE_PHILOX
    elif noise in ("reference-gpu", "reference-cpu"):
        nmode_kind = L.EEMD_NOISE_INJECTED
    else:
        raise ValueError("noise must be 'philox', 'reference-gpu' or 'reference-cpu'")
    p = make_params(dtype=dt, noise_mode=nmode_kind, eps=eps, seed=seed, tau=tau,
                    max_sifts=max_sifts, max_imf=slots, min_extrema=min_extrema, end=end,
                    rules=rules, exact=exact, config=config)
    ck = state = None
    if checkpoint is not None:
        ck = Checkpoint(checkpoint, checkpoint_key(
            x, E=E, eps=float(eps), tau=float(tau), max_sifts=int(max_sifts), max_imf=int(slots),
            min_extrema=int(min_extrema), end=end, seed=int(seed), noise=noise, rules=rules,
            exact=bool(exact), dtype=dt, config=config))
        state = ck.load()
        if state is not None:
            if batch is not None and int(batch) != int(state["batch"]):
                raise ValueError(f"checkpoint {ck.path} was written with batch={int(state['batch'])}")
            batch = int(state["batch"])  # the same batch boundaries, so the same sums
    if batch is None:
        batch = _auto_batch(torch, p, N, E, dt.itemsize)
    batch = max(1, min(int(batch), E))
    host_noise = (reference_noise(x, E, eps, seed, noise)
                  if nmode_kind == L.EEMD_NOISE_INJECTED else None)

    with nvtx.range("eemd.upload"):
        xd = torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).to(dev)
        imf_sum = torch.zeros((slots, N), dtype=torch.float64, device=dev)
        mode_count = torch.zeros((slots,), dtype=torch.int32, device=dev)
        # the per-trial sift counts, mode counts and flags of every batch in one
        # device array, copied back with the outputs (no wait between launches)
        cnt = torch.empty((3, E), dtype=torch.int32, device=dev)
        first = 0
        if state is not None:
            first = int(state["next"])
            imf_sum.copy_(torch.from_numpy(state["imf_sum"]))
            mode_count.copy_(torch.from_numpy(state["mode_count"]))
            cnt[:, :first].copy_(torch.from_numpy(state["counters"]))
    ws = None
    t0 = time.time()
    for b0 in range(first, E, batch):
        b1 = min(E, b0 + batch)
        Eb = b1 - b0
        pb = tuned(p, [N], Eb)
        need = L.workspace_size(pb, [N], Eb, False)
        if ws is None or ws.numel() < need:
            ws = torch.empty((need,), dtype=torch.uint8, device=dev)
        nz = None
        if host_noise is not None:
            nz = torch.from_numpy(np.ascontiguousarray(host_noise[b0:b1], dtype=dt)).to(dev)
        with nvtx.range("eemd.batch"):
            L.run(pb, xd, [N], b0, Eb, ws, noise=nz, imf_sum=imf_sum, mode_count=mode_count,
                  nsift=cnt[0, b0:b1], nmode=cnt[1, b0:b1], flags=cnt[2, b0:b1])
        if ck is not None:
            with nvtx.range("eemd.checkpoint"):
                ck.save(batch=batch, next_trial=b1, imf_sum=imf_sum.cpu().numpy(),
                        mode_count=mode_count.cpu().numpy(), counters=cnt[:, :b1].cpu().numpy())
    imf_mean = torch.empty((slots, N), dtype=torch.float64, device=dev)
    resid = torch.empty((N,), dtype=torch.float64, device=dev)
    n_modes_d = torch.empty((1,), dtype=torch.int32, device=dev)
    with nvtx.range("eemd.finalize"):
        L.finalize(p, xd, [N], imf_sum, mode_count, imf_mean, resid, n_modes_d)
    # all outputs through pinned memory with one synchronisation
    if slots * N * 8 <= PINNED_RESULT_BYTES:
        with nvtx.range("eemd.download"):
            h_mean, h_resid = _pinned(torch, (slots, N), torch.float64), _pinned(torch, (N,), torch.float64)
            h_n, ch = _pinned(torch, (1,), torch.int32), _pinned(torch, (3, E), torch.int32)
            h_mean.copy_(imf_mean, non_blocking=True)
            h_resid.copy_(resid, non_blocking=True)
            h_n.copy_(n_modes_d, non_blocking=True)
            ch.copy_(cnt, non_blocking=True)
            torch.cuda.current_stream(dev).synchronize()
            n_modes = int(h_n[0])
            imfs = h_mean[:n_modes].numpy()
            residual = h_resid.numpy()
    else:
        with _STAGE_LOCK, nvtx.range("eemd.download"):  # callers on several threads share the buffers
            h_mean, h_resid, h_n = _staging(torch, slots, N)
            h_mean.copy_(imf_mean, non_blocking=True)
            h_resid.copy_(resid, non_blocking=True)
            h_n.copy_(n_modes_d, non_blocking=True)
            ch = cnt.cpu()  # synchronises the stream: every copy above has landed
            n_modes = int(h_n[0])
            imfs = fresh_copy(h_mean[:n_modes].numpy())
            residual = h_resid.numpy().copy()
    per_trial_sifts, per_trial_modes, flags_all = ch[0].tolist(), ch[1].tolist(), ch[2].tolist()
    if ck is not None:
        ck.remove()
    dt_s = time.time() - t0
    reached = any(f & 1 for f in flags_all)
    stats = dict(method="gpu", backend="b200", E=E, n_modes=n_modes, batch=batch,
                 per_trial_total_sifts=np.array(per_trial_sifts),
                 per_trial_n_modes=np.array(per_trial_modes),
                 max_imf_reached=bool(reached and max_imf == -1),
                 gpu_time_s=dt_s, noise=noise if E > 1 else "none", x=np.asarray(x, dtype=float))
    return imfs, residual, stats


def _run_single(x, *, tau, max_sifts, max_imf, min_extrema, end, rules, exact, dtype, config):
    """Plain EMD (E=1): the trial's own IMFs and its sequential residual, like
    the reference's E=1 CPU path (emd_par.py:146-154)."""
    torch = _torch()
    N = len(x)
    slots = imf_slots(N, max_imf)
    dt = np.dtype(dtype)
    tdt = _tdtype(torch, dt)
    dev = torch.device("cuda", torch.cuda.current_device())
    p = make_params(dtype=dt, noise_mode=L.EEMD_NOISE_NONE, tau=tau, max_sifts=max_sifts,
                    max_imf=slots, min_extrema=min_extrema, end=end, rules=rules, exact=exact,
                    config=config)
    p = tuned(p, [N], 1)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).to(dev)
    ws = torch.empty((L.workspace_size(p, [N], 1, True),), dtype=torch.uint8, device=dev)
    # (the engine writes every IMF row it returns; the rows past the mode count are not read)
    imfs = torch.empty((1, slots, N), dtype=tdt, device=dev)
    resid = torch.empty((1, N), dtype=tdt, device=dev)
    # the counters in one array (sifts, modes, flags, sifts per mode): one copy back
    cnt = torch.empty((3 + slots,), dtype=torch.int32, device=dev)
    t0 = time.time()
    L.run(p, xd, [N], 0, 1, ws, imfs=imfs, resid_out=resid, nsift=cnt[0:1], nmode=cnt[1:2],
          mode_sifts=cnt[3:], flags=cnt[2:3])
    # every output into pinned memory, one synchronisation
    h_imfs, h_res = _pinned(torch, (slots, N), torch.float64), _pinned(torch, (N,), torch.float64)
    h_cnt = _pinned(torch, (3 + slots,), torch.int32)
    h_imfs.copy_(imfs[0].to(torch.float64), non_blocking=True)
    h_res.copy_(resid[0].to(torch.float64), non_blocking=True)
    h_cnt.copy_(cnt, non_blocking=True)
    torch.cuda.current_stream(dev).synchronize()
    c = h_cnt.tolist()
    nm = int(c[1])
    out = h_imfs[:nm].numpy()
    res = h_res.numpy()
    stats = dict(method="gpu", backend="b200", E=1, n_modes=nm, total_sifts=int(c[0]),
                 per_mode_sifts=[int(v) for v in c[3:3 + nm]], per_trial_total_sifts=np.array([int(c[0])]),
                 max_imf_reached=bool(int(c[2]) & 1 and max_imf == -1),
                 gpu_time_s=time.time() - t0, x=np.asarray(x, dtype=float))
    return out, res, stats


# =====================================================================
# Public API (emd_par.py:260-301)
# =====================================================================
def decompose(x, method="auto", E=64, eps=0.2, tau=0.25, max_sifts=50, max_imf=-1,
              min_extrema=4, end="natural", n_workers=None, seed=0, parallel=True, batch=None,
              nthreads=128, *, noise="philox", rules="ref", exact=False, dtype=np.float64,
              config: EngineConfig | None = None, checkpoint=None):
    """Decompose a 1-D signal x into IMFs (+ residual) on the B200 engine.

    Arguments follow emd_par.decompose; n_workers, parallel and nthreads are
    accepted for signature compatibility and ignored (the engine picks its own
    launch shapes).  Returns EMDResult with .imfs [n_modes, N] (float64),
    .residual [N], .n_modes and .stats.
    """
    x = np.asarray(x, dtype=float)
    if x.ndim != 1:
        raise ValueError("x must be 1-D")
    N = len(x)
    if N < 8:
        raise ValueError("signal too short for EMD (need >= 8 samples)")
    if method == "cpu":
        raise ValueError("method='cpu' is not provided by the B200 engine (no CPU backend); "
                         "use method='gpu' or 'auto'")
    if method not in ("auto", "gpu"):
        raise ValueError("method must be 'auto', 'cpu', or 'gpu'")
    E = int(E)
    if E < 1:
        raise ValueError("E must be >= 1")
    if E == 1:
        imfs, resid, stats = _run_single(x, tau=tau, max_sifts=max_sifts, max_imf=max_imf,
                                         min_extrema=min_extrema, end=end, rules=rules,
                                         exact=exact, dtype=dtype, config=config)
    else:
        imfs, resid, stats = _run_ensemble(x, E=E, eps=eps, tau=tau, max_sifts=max_sifts,
                                           max_imf=max_imf, min_extrema=min_extrema, end=end,
                                           seed=seed, batch=batch, noise=noise, rules=rules,
                                           exact=exact, dtype=dtype, config=config,
                                           checkpoint=checkpoint)
    return EMDResult(imfs=imfs, residual=resid, n_modes=imfs.shape[0], stats=stats)


def decompose_many(xs, E=64, eps=0.2, tau=0.25, max_sifts=50, max_imf=-1, min_extrema=4,
                   end="natural", seed=0, batch=None, *, rules="ref", exact=False, dtype=np.float64,
                   config: EngineConfig | None = None) -> list:
    """EEMD (E > 1) or EMD (E = 1) of many 1-D signals of any lengths: every
    (signal, trial) task of a trial batch in one persistent launch, the tasks
    queued longest first.  Returns one EMDResult per signal, as decompose
    would.  The Philox noise is keyed by (seed, signal index in xs, trial), so
    signal i's ensemble equals decompose(xs[i], seed=seed) only for i = 0;
    with E = 1 every result equals decompose(xs[i], E=1) (IMFs bit for bit;
    the residual is x minus the IMFs' sum here)."""
    xs = [np.asarray(x, dtype=float) for x in xs]
    if not xs:
        return []
    for x in xs:
        if x.ndim != 1:
            raise ValueError("every signal must be 1-D")
        if len(x) < 8:
            raise ValueError("signal too short for EMD (need >= 8 samples)")
    E = int(E)
    if E < 1:
        raise ValueError("E must be >= 1")
    torch = _torch()
    lengths = [len(x) for x in xs]
    S, NS = len(xs), sum(lengths)
    slots = imf_slots(max(lengths), max_imf)
    dt = np.dtype(dtype)
    dev = torch.device("cuda", torch.cuda.current_device())
    mode = L.EEMD_NOISE_NONE if E == 1 else L.EEMD_NOISE_PHILOX
    p = make_params(dtype=dt, noise_mode=mode, eps=eps, seed=seed, tau=tau, max_sifts=max_sifts,
                    max_imf=slots, min_extrema=min_extrema, end=end, rules=rules, exact=exact,
                    config=config)
    if batch is None:
        free, _ = torch.cuda.mem_get_info()
        per_trial = L.workspace_size(p, lengths, 1, False)
        batch = max(1, int(free * 0.7 // max(per_trial, 1)))
    batch = max(1, min(int(batch), E))
    p = tuned(p, lengths, batch)
    xd = torch.from_numpy(np.concatenate([x.astype(dt) for x in xs])).to(dev)
    imf_sum = torch.zeros((slots * NS,), dtype=torch.float64, device=dev)
    mode_count = torch.zeros((S * slots,), dtype=torch.int32, device=dev)
    ws = torch.empty((L.workspace_size(p, lengths, batch, False),), dtype=torch.uint8, device=dev)
    paged = None
    if slots * NS * 8 > PINNED_RESULT_BYTES:
        # large results: their host arrays are paged in on the copy threads while the device works
        mh_host, rh_host = np.empty((slots * NS,), dtype=np.float64), np.empty((NS,), dtype=np.float64)
        paged = (mh_host, rh_host, prefault([mh_host, rh_host]))
    sifts = np.zeros((S, E), dtype=np.int64)
    modes = np.zeros((S, E), dtype=np.int64)
    flags = np.zeros((S, E), dtype=np.int64)
    t0 = time.time()
    for b0 in range(0, E, batch):
        Eb = min(batch, E - b0)
        cnt = torch.empty((3, S * Eb), dtype=torch.int32, device=dev)
        L.run(p, xd, lengths, b0, Eb, ws, imf_sum=imf_sum, mode_count=mode_count, nsift=cnt[0], nmode=cnt[1],
              flags=cnt[2])
        ch = cnt.cpu().numpy().reshape(3, S, Eb)  # tasks are signal-major: task = s * Eb + e
        sifts[:, b0:b0 + Eb], modes[:, b0:b0 + Eb], flags[:, b0:b0 + Eb] = ch[0], ch[1], ch[2]
    imf_mean = torch.empty((slots * NS,), dtype=torch.float64, device=dev)
    resid = torch.empty((NS,), dtype=torch.float64, device=dev)
    n_modes = torch.empty((S,), dtype=torch.int32, device=dev)
    L.finalize(p, xd, lengths, imf_sum, mode_count, imf_mean, resid, n_modes)
    mh, rh, nh = _download(torch, dev, imf_mean, resid, n_modes, paged)
    wall = time.time() - t0
    # every signal's result is a view of the launch's host arrays (no per-signal copy)
    out, off = [], 0
    for s, x in enumerate(xs):
        n = lengths[s]
        m = int(nh[s])
        imfs = mh[slots * off:slots * (off + n)].reshape(slots, n)[:m]
        stats = dict(method="gpu", backend="b200", E=E, n_modes=m, batch=batch, signal=s, signals=S,
                     per_trial_total_sifts=sifts[s].copy(), per_trial_n_modes=modes[s].copy(),
                     max_imf_reached=bool((flags[s] & 1).any() and max_imf == -1), gpu_time_s=wall,
                     noise="philox" if E > 1 else "none", x=x)
        out.append(EMDResult(imfs=imfs, residual=rh[off:off + n], n_modes=m, stats=stats))
        off += n
    return out


def _download(torch, dev, imf_mean, resid, n_modes, paged):
    """The finalised means, residuals and mode counts of a batch into host
    arrays: small results through pinned tensors of the call, large ones
    through the shared pinned staging in slices, each slice copied out on the
    copy threads into fresh arrays paged in beforehand (`paged`: their
    prefault futures) while the next slice crosses."""
    nb = imf_mean.numel() * 8
    if nb <= PINNED_RESULT_BYTES:
        h_m, h_r = _pinned(torch, (imf_mean.numel(),), torch.float64), _pinned(torch, (resid.numel(),), torch.float64)
        h_n = _pinned(torch, (n_modes.numel(),), torch.int32)
        h_m.copy_(imf_mean, non_blocking=True)
        h_r.copy_(resid, non_blocking=True)
        h_n.copy_(n_modes, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return h_m.numpy(), h_r.numpy(), h_n.numpy()
    mh, rh, futs = paged
    nh = n_modes.cpu().numpy()
    with _STAGE_LOCK:
        stage = _staging(torch, 2, PINNED_RESULT_BYTES // 16)[0].reshape(-1)  # 64 MB, two halves
        half = stage.numel() // 2
        for f in futs:
            f.result()
        for dst, src in ((mh, imf_mean), (rh, resid)):
            n, marks, i0 = src.numel(), [], 0
            hs = stage.numpy()
            while i0 < n:
                i1 = min(n, i0 + half)
                buf = (len(marks) & 1) * half
                if len(marks) >= 2:  # the half this slice reuses has been copied out
                    marks[-2][2].synchronize()
                    a0, a1, _, b0 = marks[-2]
                    copy_into(dst[a0:a1], hs[b0:b0 + (a1 - a0)])
                stage[buf:buf + (i1 - i0)].copy_(src[i0:i1], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record()
                marks.append((i0, i1, ev, buf))
                i0 = i1
            for a0, a1, ev, b0 in marks[-2:]:
                ev.synchronize()
                copy_into(dst[a0:a1], hs[b0:b0 + (a1 - a0)])
    return mh, rh, nh


def gpu_eemd_full(x, E=64, tau=0.25, max_sifts=50, max_imf=12, seed=0, K=None, nthreads=128,
                  batch=None, *, rules="numba", exact=False, end="natural", min_extrema=4,
                  config: EngineConfig | None = None):
    """Raw per-trial decomposition of already perturbed signals
    (emd_gpu.py:301-334).  x: [E, N] (or [N] with E=1).
    Returns (imfs [E, max nmode, N], nsift [E], nmode [E]) as numpy arrays.
    Defaults to the numba kernel's stop rules (rules='numba')."""
    x = np.asarray(x, dtype=np.float64)
    if x.ndim == 1:
        if E != 1:
            raise ValueError(
                "1-D input x is a single trial (E=1). For E>1 pass a 2-D "
                "(E, N) array of perturbed signals, e.g. x[None,:] + noises.")
        x = x[None, :]
    E, N = x.shape
    if N < 3:
        raise ValueError("signal too short")
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    p = make_params(noise_mode=L.EEMD_NOISE_PREPERTURBED, tau=tau, max_sifts=max_sifts,
                    max_imf=int(max_imf), min_extrema=min_extrema, end=end, rules=rules,
                    exact=exact, config=config)
    p = tuned(p, [N], E)
    xd = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    out = torch.zeros((E, int(max_imf), N), dtype=torch.float64, device=dev)
    nsift = torch.zeros((E,), dtype=torch.int32, device=dev)
    nmode = torch.zeros((E,), dtype=torch.int32, device=dev)
    ws = torch.empty((L.workspace_size(p, [N], E, True),), dtype=torch.uint8, device=dev)
    L.run(p, xd, [N], 0, E, ws, imfs=out, nsift=nsift, nmode=nmode)
    nm = nmode.cpu().numpy()
    maxm = int(nm.max()) if nm.size else 0
    return out[:, :maxm].cpu().numpy(), nsift.cpu().numpy(), nm


# =====================================================================
# Reference signal (emd_par.py:307-318)
# =====================================================================
def make_reference_sweep(FS=44100, T=10.0, F1=20.0, F2=20000.0, noise_level=0.01, seed=0):
    """10-octave log sine sweep F1..F2 over T seconds at FS, plus white noise at
    noise_level (fraction of the unit peak).  Returns (x, t)."""
    N = int(FS * T)
    t = np.arange(N) / FS
    ratio = F2 / F1
    phi = 2 * np.pi * F1 * T * (ratio ** (t / T) - 1.0) / np.log(ratio)
    x = np.sin(phi)
    rng = np.random.default_rng(seed)
    x = x + noise_level * rng.standard_normal(N)
    return x, t
