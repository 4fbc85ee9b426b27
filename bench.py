#!/usr/bin/env python
"""EEMD throughput on one B200 (or N independent replicas), one JSON line.

Default workload (one "step"): full EEMD of 1 s of 48 kHz synthetic audio --
harmonic tone f0=220 Hz with 8 partials (1/k), pink noise at -30 dB, 5
decaying clicks, seed 1 -- N=48000 samples, 100 trials, Philox noise
0.2*std(x), 8 IMFs, fixed 10 sifts per IMF, float32 storage with float64
spline solve.  Metric: Msamples*trials/s = sum(N)*E / step time (whole job:
summed over ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload harmonic48k|plain8k|amfm4m|uneven512|surrogate|ceemdan48k|spectra48k]

The other workloads measure the remaining configurations of the path:
plain8k (single-trial plain EMD, float64, mirror ends, N=8192), amfm4m (N=2^22
AM/FM signal, float64, 256 trials in launches of 64, 12 IMFs, SD<0.2 capped
at 20 sifts, seam halo 30) and uneven512 (512 signals of log-uniform length
4096..262144, all 32 768 (signal, trial) tasks in one launch, 10 IMFs, float32
storage; the line also times the same work as one launch per signal).

--impl reference times the reference's CPU algorithm (the numpy port in
oracle/, emd_ref.py semantics, float64) on the host cores with a spawn process
pool, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "EEMD Msamples*trials/s"
UNIT = "Msamples*trials/s"
L2_BYTES = 126 * 1024 * 1024


@dataclass
class Workload:
    name: str
    config: dict
    E: int
    eps: float
    max_imf: int
    max_sifts: int
    tau: float            # SD threshold; 0 never holds, so every IMF takes max_sifts sifts
    dtype: str            # "f32" or "f64" storage (the spline solve is float64 either way)
    seed: int
    end: str = "natural"
    halo: int = 0         # seam-window halo (0: the engine's default)
    trial_batch: int = 0  # trials per launch (0: all at once)
    per_signal: bool = False  # also time the same work as one launch sequence per signal
    cpu_tasks: int = 0        # CPU-baseline sample: tasks (0: one per core, at most 32)
    cpu_max_imf: int = 0      # CPU-baseline sample: IMFs per task (0: all)
    cpu_max_sifts: int = 0    # CPU-baseline sample: sift cap (0: the workload's)
    signals_fn: object = None
    _signals: list = field(default=None, repr=False)

    def signals(self) -> list:
        if self._signals is None:
            self._signals = [np.asarray(s, dtype=np.float64) for s in self.signals_fn()]
        return self._signals

    @property
    def np_dtype(self):
        return np.float32 if self.dtype == "f32" else np.float64


def _harmonic():
    from eemd4cuda_b200 import signals
    return [signals.harmonic_clicks(48000, seed=1)]


def _plain8k():
    from eemd4cuda_b200 import signals
    return [signals.plain_emd_8k()]


def _amfm():
    from eemd4cuda_b200 import signals
    return [signals.amfm_long(1 << 22, seed=2)]


def _uneven():
    from eemd4cuda_b200 import signals
    return signals.uneven_batch(512, seed=4)


WORKLOADS = {
    "harmonic48k": Workload(
        "harmonic48k",
        {"workload": "harmonic_clicks_48k_eemd", "N": 48000, "trials": 100, "eps": 0.2,
         "max_imf": 8, "sifts_per_imf": 10, "storage": "float32", "solve": "float64",
         "noise": "philox", "signals": 1},
        E=100, eps=0.2, max_imf=8, max_sifts=10, tau=0.0, dtype="f32", seed=1,
        signals_fn=_harmonic),
    "plain8k": Workload(
        "plain8k",
        {"workload": "plain_emd_8k", "N": 8192, "trials": 1, "max_imf": 10, "tau": 0.2,
         "max_sifts": 10, "ends": "mirror", "storage": "float64", "solve": "float64",
         "signals": 1},
        E=1, eps=0.0, max_imf=10, max_sifts=10, tau=0.2, dtype="f64", seed=0, end="mirror",
        cpu_tasks=8, signals_fn=_plain8k),
    "amfm4m": Workload(
        "amfm4m",
        {"workload": "amfm_2^22_eemd", "N": 1 << 22, "trials": 256, "eps": 0.2, "max_imf": 12,
         "tau": 0.2, "max_sifts": 20, "storage": "float64", "solve": "float64",
         "seam_halo": 30, "knots_per_block": 5, "noise": "philox", "signals": 1, "trials_per_launch": 64},
        E=256, eps=0.2, max_imf=12, max_sifts=20, tau=0.2, dtype="f64", seed=2, halo=30,
        trial_batch=64, cpu_tasks=16, cpu_max_imf=1, cpu_max_sifts=2, signals_fn=_amfm),
    "uneven512": Workload(
        "uneven512",
        {"workload": "uneven_512_signals_eemd", "signals": 512,
         "lengths": "log-uniform 4096..262144", "trials": 64, "eps": 0.2, "max_imf": 10,
         "sifts_per_imf": 10, "storage": "float32", "solve": "float64", "noise": "philox",
         "trials_per_launch": 64},
        E=64, eps=0.2, max_imf=10, max_sifts=10, tau=0.0, dtype="f32", seed=1, trial_batch=0,
        per_signal=True, cpu_tasks=32, signals_fn=_uneven),
}


def rank_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


# ---------------------------------------------------------------------------
# CPU side: the reference's own CPU code (baseline/_ref), else the numpy port
# ---------------------------------------------------------------------------
REF_DIR = ROOT / "baseline" / "_ref"


def reference_installed() -> bool:
    return (REF_DIR / "emd_ref.py").exists() and (REF_DIR / "emd_par.py").exists()


def _ref_trial(args):
    """One trial of the reference's CPU EEMD, run by the reference's own code:
    emd_ref.emd_1d of the unmodified reference installed in baseline/_ref, on
    x + the reference CPU path's per-trial noise (emd_par.py:112-119: numpy
    default_rng((seed * 1000003 + e) mod 2^64), standard normals times
    eps*std(x)); no noise for plain EMD (emd_par.py:148-151)."""
    x, seed, e, sigma, kw = args
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    import emd_ref
    t0 = time.perf_counter()
    if sigma > 0:
        rng = np.random.default_rng((seed * 1000003 + e) & 0xFFFFFFFFFFFFFFFF)
        x = x + rng.standard_normal(len(x)) * sigma
    imfs, resid, st = emd_ref.emd_1d(x, **kw)
    return len(imfs), st["total_sifts"], time.perf_counter() - t0


class CpuBaseline:
    """The reference's CPU algorithm on (signal, trial) tasks of the workload
    in a spawn process pool with dynamic scheduling.

    kind "reference": the reference's own emd_ref.emd_1d (baseline/_ref) with
    the reference CPU path's noise stream, as emd_par._cpu_decompose runs it
    (emd_par.py:139-183); the pool passes max_imf on, which the stock ensemble
    path does not (emd_par.py:118-119 drops it, so decompose(method='cpu',
    E>1) would decompose every mode rather than the workload's).  kind
    "port": the numpy restatement in oracle/ when the reference is not
    installed.  The sample is a bounded set of tasks (float64) so that one
    step takes seconds.  With cpu_max_imf / cpu_max_sifts the sample runs
    only the first sifts, and `value` scales the time per sift to a full
    task's sift count."""

    def __init__(self, wl: Workload):
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor

        self.wl = wl
        self.kind = "reference" if reference_installed() else "port"
        self.cores = 1 if wl.E == 1 else (os.cpu_count() or 1)
        sig = wl.signals()
        rng = np.random.default_rng(wl.seed)
        n_tasks = wl.cpu_tasks or max(4, min(self.cores, 32))
        self.kw = dict(tau=wl.tau, max_sifts=wl.cpu_max_sifts or wl.max_sifts,
                       max_imf=wl.cpu_max_imf or wl.max_imf, end=wl.end)
        self.tasks = []
        for e in range(n_tasks):
            s = int(rng.integers(len(sig))) if len(sig) > 1 else 0
            x = sig[s].astype(wl.np_dtype).astype(np.float64)
            sigma = wl.eps * np.std(x) if wl.E > 1 else 0.0
            if self.kind == "reference":
                self.tasks.append((x, wl.seed, e, sigma, self.kw))
            else:
                noise = rng.standard_normal(len(x)) * sigma if wl.E > 1 else np.zeros(len(x))
                self.tasks.append((x, noise, self.kw))
        self.pool = ProcessPoolExecutor(max_workers=self.cores, mp_context=mp.get_context("spawn"))
        self.sifts_done = 0
        self.full_sifts = None

    def step(self) -> float:
        from concurrent.futures import as_completed
        from oracle import emd_oracle as O

        fn = _ref_trial if self.kind == "reference" else O._trial_worker
        t0 = time.perf_counter()
        futs = [self.pool.submit(fn, t) for t in self.tasks]
        sifts = 0
        for f in as_completed(futs):
            sifts += f.result()[1]
        self.sifts_done = sifts
        return time.perf_counter() - t0

    def value(self, seconds: float, full_sifts_per_task: float | None = None) -> float:
        samples = sum(len(t[0]) for t in self.tasks)
        if self.wl.cpu_max_imf or self.wl.cpu_max_sifts:
            self.full_sifts = full_sifts_per_task or self.wl.max_imf * self.wl.max_sifts / 2
            seconds *= self.full_sifts / max(self.sifts_done / len(self.tasks), 1e-9)
        return samples / seconds / 1e6

    def describe(self, v: float) -> dict:
        wl = self.wl
        who = ("the reference's own emd_ref.emd_1d (unmodified, installed in baseline/_ref) with its "
               "CPU path's per-trial noise stream" if self.kind == "reference"
               else "emd_1d of the numpy restatement in oracle/")
        what = (f"{len(self.tasks)} (signal, trial) tasks of the workload ({who}, float64 "
                f"arithmetic on the workload's {'float32-rounded ' if wl.dtype == 'f32' else ''}signal, "
                f"tau={wl.tau}, max_sifts={self.kw['max_sifts']}, max_imf={self.kw['max_imf']}, "
                f"{wl.end} ends) in a {self.cores}-process pool with dynamic scheduling")
        if wl.cpu_max_imf or wl.cpu_max_sifts:
            what += (f"; the time per sift of IMF 1 scaled to {self.full_sifts:.1f} sifts per task "
                     "(IMF-1 sifts are the slowest, so this bounds the CPU time from above)")
        return {"value": round(v, 4), "unit": UNIT, "cores": self.cores, "kind": self.kind,
                "sample": what}

    def close(self):
        self.pool.shutdown()


def run_reference(args, wl: Workload, metric: str = None, config: dict = None):
    """The reference's CPU algorithm (the oracle port) on a bounded sample of
    the workload, on all host cores; `metric` and `config` default to the
    EEMD workload's and are passed where the GPU arm names its line
    differently (CEEMDAN, the surrogate)."""
    rank, _, world = rank_env()
    if rank != 0:
        return 0
    cb = CpuBaseline(wl)
    big = wl.name in ("amfm4m", "uneven512")
    steps = max(1, min(args.steps, 2)) if big else args.steps
    warm = 1 if big else args.warmup
    for _ in range(warm):
        cb.step()
    ts = [cb.step() for _ in range(steps)]
    cb.close()
    sec = sum(ts) / len(ts)
    v = cb.value(sec)
    # the workload as the GPU arm names it, with what this arm actually runs:
    # float64 storage and arithmetic, the reference CPU path's noise stream, a
    # bounded sample of tasks (cpu_baseline.sample)
    cfg = dict(config) if config is not None else dict(wl.config)
    if "storage" in cfg:
        cfg["storage"] = "float64"
    if "noise" in cfg:
        cfg["noise"] = ("numpy default_rng per trial (the reference CPU path's stream, emd_par.py:112-119)"
                        if cb.kind == "reference" else "numpy default_rng")
    cfg["tasks_per_step"] = len(cb.tasks)
    line = {"impl": "reference", "metric": metric or METRIC, "value": round(v, 4), "unit": UNIT,
            "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": cb.describe(v),
            "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons sampled every 10 ms during the timed
    region (NVML; nvidia-smi at 200 ms when NVML is unavailable)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples: list[tuple[float, float, int]] = []
        self.stop_evt = threading.Event()
        self.thread = None
        self.nvml = None

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.nvml = (nv, h)
        except Exception:
            self.nvml = None
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        if self.nvml is not None:
            nv, h = self.nvml
            getr = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            while not self.stop_evt.is_set():
                try:
                    self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                         float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)),
                                         int(getr(h))))
                except Exception:
                    break
                self.stop_evt.wait(0.01)
            return
        try:
            proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.active", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        while not self.stop_evt.is_set():
            line = proc.stdout.readline()
            if not line:
                break
            parts = [q.strip() for q in line.split(",")]
            try:
                self.samples.append((float(parts[0]), float(parts[1]), int(parts[2], 16)))
            except (ValueError, IndexError):
                pass
        proc.terminate()

    def stop(self) -> dict:
        self.stop_evt.set()
        if self.thread:
            self.thread.join(timeout=5)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        reasons = sorted(k for k, bit in self.REASONS.items()
                         if any(r & bit for _, _, r in self.samples))
        return {"sm_mhz": statistics.median(s for s, _, _ in self.samples),
                "sm_max_mhz": max(m for _, m, _ in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": "nvml" if self.nvml else "nvidia-smi"}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


# DRAM traffic of one k_emd launch: ncu dram__bytes_read.sum +
# dram__bytes_write.sum from a capture of the same workload (a capture cannot
# run inside the timed bench).  `engine_sha256` is the hash of the engine
# source the capture ran; the bench reports whether the current source is the
# same (`traffic_matches_build`), so a change of the kernel since the capture
# shows.  Workloads too large to capture whole were captured on fewer trials
# of the same signal and are scaled per (signal, trial) task, since every task
# streams its own buffers.
EMD_TRAFFIC = {
    "harmonic48k": {"bytes_per_launch": 6837855000,
                    "engine_sha256": "3788a361741c024d3ab67bed60b11685f8a5f528f948919fb8eb3f3ad6b353ab",
                    "capture": "one k_emd launch of the 100-trial 48 kHz workload (clusters of 4 five-warp CTAs)"},
    "amfm4m": {"bytes_per_task": 5603181376.0,
               "engine_sha256": "3788a361741c024d3ab67bed60b11685f8a5f528f948919fb8eb3f3ad6b353ab",
               "capture": "one k_emd launch of 4 trials of the 2^22-sample signal (clusters of 16 four-warp "
                          "CTAs), per task"},
}


def engine_source_sha256() -> str:
    import hashlib
    src = ROOT / "eemd4cuda_b200" / "csrc" / "eemd_engine.cu"
    return hashlib.sha256(src.read_bytes()).hexdigest()


def measured_traffic(workload: str, tasks_per_launch: int):
    """(DRAM bytes of one k_emd launch, description) from EMD_TRAFFIC, or
    (None, None) when the workload has no capture."""
    ent = EMD_TRAFFIC.get(workload)
    if not ent:
        return None, None
    b = ent.get("bytes_per_launch")
    if b is None:
        b = ent["bytes_per_task"] * tasks_per_launch
    src = {"capture": ent["capture"], "engine_sha256": ent["engine_sha256"],
           "traffic_matches_build": ent["engine_sha256"] == engine_source_sha256()}
    return int(round(b)), src


def emd_algorithmic_bytes(klog: np.ndarray, nmode: np.ndarray, lengths, trials: int,
                          bytes_el: int) -> float:
    """Algorithmic bytes of one k_emd launch, from the per-sift knot log.

    Per task of a signal of n samples (b bytes per sample; P = maxima + minima
    knots of a sift): per sift 3*n*b + P*(3*(4+b) + 2*8) -- extrema pass
    (reads h, writes the knots), solve (reads the knots, writes the second
    derivatives), evaluation pass (reads and writes h, reads knots and second
    derivatives); per IMF 4*n*b (residual read and write, IMF read, the next
    count's read); per task 2*n*b (input read, perturbed-input write).  The
    float64 ensemble accumulator belongs to k_reduce and is not counted."""
    total = 0.0
    kb = 4 + bytes_el
    for t in range(klog.shape[0]):
        n = int(lengths[t // trials])
        total += 2 * n * bytes_el
        for m in range(int(nmode[t])):
            for k in range(klog.shape[2]):
                a, b = klog[t, m, k]
                if a < 0:
                    break
                total += 3 * n * bytes_el + (int(a) + int(b)) * (3 * kb + 16)
            total += 4 * n * bytes_el
    return total


class Engine:
    """Device buffers and one EEMD step of a workload (all signals, all trials)."""

    def __init__(self, wl: Workload, dev, seed: int, signals=None):
        import torch
        from eemd4cuda_b200 import _lib as L
        from eemd4cuda_b200 import emd_par as M

        self.L, self.wl = L, wl
        sig = signals if signals is not None else wl.signals()
        self.lengths = [len(s) for s in sig]
        self.n_total = sum(self.lengths)
        noise = L.EEMD_NOISE_PHILOX if wl.E > 1 else L.EEMD_NOISE_NONE
        cfg = M.EngineConfig(halo=wl.halo) if wl.halo else None
        self.batch = wl.trial_batch or wl.E
        # the product's launch choice: the autotune table's threads per trial
        self.p = M.tuned(M.make_params(dtype=wl.np_dtype, noise_mode=noise, eps=wl.eps, seed=seed,
                                       tau=wl.tau, max_sifts=wl.max_sifts, max_imf=wl.max_imf, end=wl.end,
                                       config=cfg), self.lengths, self.batch)
        self.host = np.concatenate([s.astype(wl.np_dtype) for s in sig])
        self.xd = torch.from_numpy(self.host).to(dev)
        self.ws = torch.empty((L.workspace_size(self.p, self.lengths, self.batch, False),),
                              dtype=torch.uint8, device=dev)
        m = wl.max_imf
        self.imf_sum = torch.zeros((m * self.n_total,), dtype=torch.float64, device=dev)
        self.mode_count = torch.zeros((len(sig) * m,), dtype=torch.int32, device=dev)
        self.imf_mean = torch.empty((m * self.n_total,), dtype=torch.float64, device=dev)
        self.resid = torch.empty((self.n_total,), dtype=torch.float64, device=dev)
        self.n_modes = torch.empty((len(sig),), dtype=torch.int32, device=dev)

    def step(self, times=None, klog=None, nmode=None, nsift=None):
        self.imf_sum.zero_()
        self.mode_count.zero_()
        for b0 in range(0, self.wl.E, self.batch):
            eb = min(self.batch, self.wl.E - b0)
            first = b0 == 0
            self.L.run(self.p, self.xd, self.lengths, b0, eb, self.ws, imf_sum=self.imf_sum,
                       mode_count=self.mode_count, times=times if first else None,
                       knot_log=klog if first else None, nmode=nmode if first else None,
                       nsift=nsift if first else None)
        self.L.finalize(self.p, self.xd, self.lengths, self.imf_sum, self.mode_count,
                        self.imf_mean, self.resid, self.n_modes)

    def launch_batches(self) -> int:
        return (self.wl.E + self.batch - 1) // self.batch


class PerSignal:
    """The same work as plain per-signal calls: for each signal in turn one
    launch of all its trials and its mean (one workspace and output set,
    sized for the longest signal, reused signal after signal)."""

    def __init__(self, wl: Workload, dev, seed: int):
        import torch
        from eemd4cuda_b200 import _lib as L
        from eemd4cuda_b200 import emd_par as M

        self.L, self.wl = L, wl
        sig = wl.signals()
        self.lengths = [len(s) for s in sig]
        self.offsets = np.concatenate([[0], np.cumsum(self.lengths)])
        cfg = M.EngineConfig(halo=wl.halo) if wl.halo else None
        base = M.make_params(dtype=wl.np_dtype, noise_mode=L.EEMD_NOISE_PHILOX, eps=wl.eps, seed=seed,
                             tau=wl.tau, max_sifts=wl.max_sifts, max_imf=wl.max_imf, end=wl.end, config=cfg)
        self.ps = [M.tuned(base, [n], wl.E) for n in self.lengths]
        self.xd = torch.from_numpy(np.concatenate([s.astype(wl.np_dtype) for s in sig])).to(dev)
        need = max(L.workspace_size(p, [n], wl.E, False) for p, n in zip(self.ps, self.lengths))
        self.ws = torch.empty((need,), dtype=torch.uint8, device=dev)
        nmax, m = max(self.lengths), wl.max_imf
        self.imf_sum = torch.zeros((m * nmax,), dtype=torch.float64, device=dev)
        self.mode_count = torch.zeros((m,), dtype=torch.int32, device=dev)
        self.imf_mean = torch.empty((m * nmax,), dtype=torch.float64, device=dev)
        self.resid = torch.empty((nmax,), dtype=torch.float64, device=dev)
        self.n_modes = torch.empty((1,), dtype=torch.int32, device=dev)

    def step(self):
        m = self.wl.max_imf
        for p, n, o in zip(self.ps, self.lengths, self.offsets):
            x = self.xd[int(o):int(o) + n]
            self.imf_sum[:m * n].zero_()
            self.mode_count.zero_()
            self.L.run(p, x, [n], 0, self.wl.E, self.ws, imf_sum=self.imf_sum, mode_count=self.mode_count)
            self.L.finalize(p, x, [n], self.imf_sum, self.mode_count, self.imf_mean, self.resid, self.n_modes)


def accuracy_check(wl: Workload, dev, pool, seed: int) -> dict:
    """Error of the engine against the float64 CPU oracle (emd_ref.py's
    algorithm, oracle/emd_oracle.py) on identical trial inputs: the
    workload's Philox noise for a few trials is drawn on the device, the
    perturbed inputs are rounded to the storage type, and both sides
    decompose exactly those rows with the workload's settings (the engine in
    its default fast mode, as timed).  Runs outside the timed region; the
    oracle is the checker here, never the thing measured."""
    import torch
    from eemd4cuda_b200 import _lib as L
    from eemd4cuda_b200 import emd_par as M
    from oracle import emd_oracle as O

    sig = wl.signals()
    max_imf, max_sifts, tau = wl.max_imf, wl.max_sifts, wl.tau
    if wl.name == "uneven512":
        picks, trials, scope = sorted(range(len(sig)), key=lambda i: len(sig[i]))[:4], 1, \
            "full decomposition of trial 0 of the 4 shortest signals"
    elif wl.name == "amfm4m":
        # a full float64 oracle decomposition of 2^22 samples takes hours on one core
        picks, trials, max_imf, max_sifts = [0], 1, 1, 2
        scope = "first 2 sifts of IMF 1 of trial 0 (the float64 oracle runs about 5 s per sift here)"
    else:
        picks, trials = [0], (4 if wl.E > 1 else 1)
        scope = f"full decomposition of trials 0..{trials - 1}"
    rows, keys = [], []
    for s in picks:
        x = sig[s].astype(wl.np_dtype).astype(np.float64)
        for e in range(trials):
            if wl.E > 1:
                nz = torch.empty((len(x),), dtype=torch.float64, device=dev)
                L.philox_normals(seed, s, e, 1, len(x), nz)
                row = x + wl.eps * np.std(x) * nz.cpu().numpy()
            else:
                row = x
            rows.append(row.astype(wl.np_dtype))
            keys.append((s, e))
    cfg = M.EngineConfig(halo=wl.halo) if wl.halo else None
    p = M.make_params(dtype=wl.np_dtype, noise_mode=L.EEMD_NOISE_PREPERTURBED, tau=tau,
                      max_sifts=max_sifts, max_imf=max_imf, end=wl.end, config=cfg)
    lengths = [len(r) for r in rows]
    tdt = torch.float32 if wl.dtype == "f32" else torch.float64
    xd = torch.from_numpy(np.concatenate(rows)).to(dev)
    imfs = torch.zeros((max_imf * sum(lengths),), dtype=tdt, device=dev)
    nmode = torch.zeros((len(rows),), dtype=torch.int32, device=dev)
    klog = torch.full((len(rows), max_imf, max_sifts, 2), -1, dtype=torch.int32, device=dev)
    ws = torch.empty((L.workspace_size(p, lengths, 1, True),), dtype=torch.uint8, device=dev)
    L.run(p, xd, lengths, 0, 1, ws, imfs=imfs, nmode=nmode, knot_log=klog)
    im = imfs.double().cpu().numpy()
    nm = nmode.cpu().numpy()
    kl = klog.cpu().numpy()
    del ws, imfs, xd
    kw = dict(tau=tau, max_sifts=max_sifts, max_imf=max_imf, end=wl.end)
    ref = list(pool.map(O._imfs_worker, [(r.astype(np.float64), kw) for r in rows]))
    per_imf = np.zeros(max_imf)
    stack, same, total, modes_equal, off = 0.0, 0, 0, True, 0
    for i, (r, (o, olog)) in enumerate(zip(rows, ref)):
        n = len(r)
        g = im[off:off + max_imf * n].reshape(max_imf, n)
        off += max_imf * n
        modes_equal = modes_equal and int(nm[i]) == len(o)
        m = min(int(nm[i]), len(o))
        for k in range(m):
            den = np.linalg.norm(o[k])
            if den > 0:
                per_imf[k] = max(per_imf[k], float(np.linalg.norm(g[k] - o[k]) / den))
        stack = max(stack, float(np.linalg.norm(g[:m] - o[:m]) / np.linalg.norm(r.astype(np.float64))))
        for mm, mode in enumerate(olog):
            for k, ab in enumerate(mode):
                total += 1
                same += int(mm < max_imf and kl[i, mm, k].tolist() == list(ab))
    return {"reference": "float64 CPU oracle (emd_ref.py algorithm) on the same storage-rounded trial inputs",
            "scope": scope, "trials_checked": len(rows),
            "max_rel_l2_vs_fp64_oracle": float(per_imf.max()),
            "max_rel_l2_per_imf": [float(f"{v:.3e}") for v in per_imf],
            "stack_rel_l2_vs_fp64_oracle": float(f"{stack:.3e}"),
            "mode_counts_equal": bool(modes_equal),
            "sifts_with_identical_knot_counts": f"{same}/{total}"}


def run_ours(args, wl: Workload):
    import torch

    rank, local_rank, world = rank_env()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=dev)

    from eemd4cuda_b200 import emd_par as M

    # the CPU baseline pool is started before any GPU work (spawn context)
    cb = CpuBaseline(wl) if (rank == 0 and world == 1 and not args.quick) else None

    eng = Engine(wl, dev, wl.seed + rank)
    L = eng.L
    flush = torch.empty((2 * L2_BYTES,), dtype=torch.uint8, device=dev)
    samples_trials = eng.n_total * wl.E

    for _ in range(args.warmup):
        eng.step()
    torch.cuda.synchronize()

    # ---- timed region: K steps, device time per step with CUDA events ----
    clk = ClockSampler(local_rank)
    clk.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    stream = torch.cuda.current_stream()
    for _ in range(args.steps):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.step()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = clk.stop()
    ms = total_ms / args.steps
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * samples_trials / (ms / 1e3) / 1e6

    # ---- per-kernel split (traced step: event pair around every launch of the first batch) ----
    times = L.KernelTimes()
    n_first = len(eng.lengths) * eng.batch
    klog = torch.full((n_first, wl.max_imf, wl.max_sifts, 2), -1, dtype=torch.int32, device=dev)
    nmode = torch.zeros((n_first,), dtype=torch.int32, device=dev)
    nsift = torch.zeros((n_first,), dtype=torch.int32, device=dev)
    flush.fill_(1)
    eng.step(times=times, klog=klog, nmode=nmode, nsift=nsift)
    torch.cuda.synchronize()
    kt = times.as_dict()
    launches_per_step = sum(v["launches"] for v in kt.values()) * eng.launch_batches() + 1
    ev = kt["emd"]
    bytes_el = 4 if wl.dtype == "f32" else 8
    emd_bytes = emd_algorithmic_bytes(klog.cpu().numpy(), nmode.cpu().numpy(), eng.lengths,
                                      eng.batch, bytes_el)
    emd_gbs = emd_bytes / (ev["ms"] / 1e3) / 1e9 if ev["ms"] > 0 else 0.0
    gpu_sifts_per_task = float(nsift.float().mean().item())
    peak, peak_kind = measured_peak_hbm()
    traffic, traffic_src = measured_traffic(wl.name, n_first)

    # ---- end to end through the public API (host buffers) ----
    if wl.name in ("harmonic48k", "plain8k"):
        x = wl.signals()[0].astype(wl.np_dtype)
        cfg = M.EngineConfig(halo=wl.halo) if wl.halo else None

        def e2e_call():
            r = M.decompose(x, E=wl.E, eps=wl.eps, tau=wl.tau, max_sifts=wl.max_sifts,
                            max_imf=wl.max_imf, seed=wl.seed + rank, end=wl.end,
                            dtype=wl.np_dtype, config=cfg)
            return r.n_modes
        h2d = x.nbytes
        e2e_warm = args.warmup
    else:
        # the batched C ABI: pinned host input in, ensemble means and residuals out
        pin_in = torch.from_numpy(eng.host).pin_memory()
        pin_out = torch.empty((wl.max_imf * eng.n_total,), dtype=torch.float64).pin_memory()
        pin_res = torch.empty((eng.n_total,), dtype=torch.float64).pin_memory()

        def e2e_call():
            eng.xd.copy_(pin_in, non_blocking=True)
            eng.step()
            pin_out.copy_(eng.imf_mean, non_blocking=True)
            pin_res.copy_(eng.resid, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            return wl.max_imf
        h2d = eng.host.nbytes
        e2e_warm = 1

    for _ in range(e2e_warm):
        e2e_call()
    torch.cuda.synchronize()
    # host-side Python and copies make single calls noisier than device steps:
    # the median of at least 20 calls (each ~10 ms), with the host clock beside
    e2e_ms, e2e_wall = [], []
    n_modes_e2e = wl.max_imf
    for _ in range(3 if args.quick else max(args.steps, 20)):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        n_modes_e2e = e2e_call()
        e1.record(stream)
        e1.synchronize()
        e2e_wall.append((time.perf_counter() - t0) * 1e3)
        e2e_ms.append(e0.elapsed_time(e1))
    e2e = statistics.median(e2e_ms)
    if dist:
        t = torch.tensor([e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())
    e2e_value = world * samples_trials / (e2e / 1e3) / 1e6
    d2h = n_modes_e2e * eng.n_total * 8 + eng.n_total * 8
    if wl.name in ("harmonic48k", "plain8k"):
        d2h += 3 * wl.E * 4  # per-trial sift, mode and flag counters

    # ---- the same work as one launch sequence per signal ----
    per_signal = None
    if wl.per_signal and rank == 0 and not args.quick:
        ps = PerSignal(wl, dev, wl.seed + rank)
        ps.step()
        torch.cuda.synchronize()
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ps.step()
        e1.record(stream)
        e1.synchronize()
        ps_ms = e0.elapsed_time(e1)
        per_signal = {"ms_per_step": round(ps_ms, 3),
                      "value": round(samples_trials / (ps_ms / 1e3) / 1e6, 3),
                      "launch_sequences": len(ps.lengths),
                      "what": "one launch of all trials per signal (the product's tuned choice for a "
                              "single-signal launch), then its mean, signal after signal",
                      "batched_speedup": round(ps_ms / ms, 3)}
        del ps
        torch.cuda.empty_cache()

    # ---- float64 storage beside the float32 headline (the reference's own precision) ----
    f64_line = None
    if wl.dtype == "f32" and wl.name == "harmonic48k" and not args.quick:
        wl64 = dataclasses.replace(wl, dtype="f64", _signals=wl.signals())
        eng64 = Engine(wl64, dev, wl.seed + rank)
        for _ in range(args.warmup):
            eng64.step()
        torch.cuda.synchronize()
        ms64 = 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng64.step()
            e1.record(stream)
            e1.synchronize()
            ms64 += e0.elapsed_time(e1)
        ms64 /= args.steps
        t64 = L.KernelTimes()
        kl64 = torch.full((n_first, wl.max_imf, wl.max_sifts, 2), -1, dtype=torch.int32, device=dev)
        nm64 = torch.zeros((n_first,), dtype=torch.int32, device=dev)
        flush.fill_(1)
        eng64.step(times=t64, klog=kl64, nmode=nm64)
        torch.cuda.synchronize()
        ev64 = t64.as_dict()["emd"]
        b64 = emd_algorithmic_bytes(kl64.cpu().numpy(), nm64.cpu().numpy(), eng64.lengths, eng64.batch, 8)
        gbs64 = b64 / (ev64["ms"] / 1e3) / 1e9 if ev64["ms"] > 0 else 0.0
        f64_line = {"dtype": "f64", "value": round(world * samples_trials / (ms64 / 1e3) / 1e6, 3),
                    "unit": UNIT, "ms_per_step": round(ms64, 4),
                    "roofline": {"kernel": "k_emd", "achieved": round(gbs64, 2), "peak": peak,
                                 "unit": "GB/s", "frac": round(gbs64 / peak, 4),
                                 "algorithmic_bytes_per_launch": round(b64 / max(ev64["launches"], 1)),
                                 "avg_launch_ms": round(ev64["ms"] / max(ev64["launches"], 1), 5)}}
        del eng64
        torch.cuda.empty_cache()

    # ---- error against the float64 CPU oracle (rank 0, outside the timed region) ----
    accuracy, acc64 = None, None
    if rank == 0 and not args.quick:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        pool = cb.pool if cb is not None else ProcessPoolExecutor(
            max_workers=min(8, os.cpu_count() or 1), mp_context=mp.get_context("spawn"))
        accuracy = accuracy_check(wl, dev, pool, wl.seed + rank)
        if f64_line is not None:
            acc64 = accuracy_check(dataclasses.replace(wl, dtype="f64", _signals=wl.signals()), dev, pool,
                                   wl.seed + rank)
            f64_line["accuracy"] = acc64
        if cb is None:
            pool.shutdown()

    cpu = None
    if cb is not None:
        cb.step()  # warm the pool's imports
        cs = cb.step()
        cpu = cb.describe(cb.value(cs, gpu_sifts_per_task))
        cb.close()

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    config = dict(wl.config, parallelism=f"replicas{world}",
                  l2="flushed between timed steps (256 MiB write)")
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype,
        "data": "synthetic", "config": config,
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "ms_per_step": round(e2e, 4),
                "calls": len(e2e_ms), "host_wall_ms": round(statistics.median(e2e_wall), 4),
                "min_ms": round(min(e2e_ms), 4),
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "kernel": "k_emd", "achieved": round(emd_gbs, 2),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(emd_gbs / peak, 4),
                     "traffic": traffic, "traffic_source": traffic_src,
                     "algorithmic_bytes_per_launch": round(emd_bytes / max(ev["launches"], 1)),
                     "avg_launch_ms": round(ev["ms"] / max(ev["launches"], 1), 5)},
        "kernel_split_ms": {k: round(v["ms"], 4) for k, v in kt.items()},
        "kernel_launches": {k: v["launches"] for k, v in kt.items()},
        "clocks": clocks,
    }
    if per_signal is not None:
        line["per_signal_launches"] = per_signal
    if accuracy is not None:
        line["accuracy"] = accuracy
    if f64_line is not None:
        line["float64_storage"] = f64_line
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if wl.name == "harmonic48k" and world == 1 and not args.quick and not args.no_companions:
        line["other_configs"] = run_companions()
    print(json.dumps(line), flush=True)
    return 0


# the other configurations, measured briefly beside the headline line (each in
# a process of its own: one timed step after 3 warm-up steps, 3 end-to-end
# calls, no CPU baseline and no oracle comparison; `--workload W` gives the
# full line of each)
COMPANIONS = (("plain8k", 180), ("amfm4m", 300), ("uneven512", 400), ("surrogate", 400), ("ceemdan48k", 180),
              ("spectra48k", 180))


def companion_summary(line: dict) -> dict:
    out = {"metric": line.get("metric"), "value": line.get("value"), "unit": line.get("unit"),
           "ms_per_step": line.get("ms_per_step"), "steps": line.get("steps"), "dtype": line.get("dtype"),
           "workload": (line.get("config") or {}).get("workload")}
    e2e = line.get("e2e")
    if isinstance(e2e, dict):
        out["e2e"] = e2e.get("value")
    rf = line.get("roofline") or {}
    out["roofline"] = {k: rf.get(k) for k in ("kernel", "achieved", "peak", "unit", "frac")}
    for k in ("roofline_hbm", "split_ms", "speedup_vs_plain_256"):
        if k in line:
            out[k] = line[k]
    out["clocks_sm_mhz"] = (line.get("clocks") or {}).get("sm_mhz")
    return out


def run_companions() -> dict:
    res = {}
    for w, limit in COMPANIONS:
        cmd = [sys.executable, str(Path(__file__).resolve()), "--workload", w, "--steps", "1", "--warmup", "3",
               "--quick"]
        env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE")}
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=limit, cwd=str(ROOT), env=env)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            if r.returncode != 0 or not lines:
                tail = (r.stderr or r.stdout).strip().splitlines()[-1:] or ["no output"]
                res[w] = {"error": f"exit {r.returncode}: {tail[0][:200]}"}
            else:
                res[w] = companion_summary(json.loads(lines[-1]))
        except subprocess.TimeoutExpired:
            res[w] = {"error": f"no line within {limit} s"}
        except Exception as e:  # a companion never takes the headline line down
            res[w] = {"error": f"{type(e).__name__}: {e}"[:200]}
    return res


# ---------------------------------------------------------------------------
# the learned surrogate (8-trial ensemble + network in place of 256 trials)
# ---------------------------------------------------------------------------
SURROGATE_WEIGHTS = ROOT / "eemd4cuda_b200" / "weights" / "surrogate_n65536.npz"
SG_SIGNALS = 128


def measured_peak_bf16():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["bf16_tflops"]), "measured"
        except (KeyError, ValueError):
            pass
    return 1590.0, "fallback"


def _surrogate_signal():
    from eemd4cuda_b200 import surrogate as SU
    return SU.make_signals([30000], 65536)


SURROGATE_METRIC = "surrogate EEMD Msamples*trials/s (256-trial equivalent)"
CEEMDAN_METRIC = "CEEMDAN Msamples*trials/s (per stage)"


def surrogate_config(weights: str) -> dict:
    """The surrogate workload as both arms name it."""
    from eemd4cuda_b200 import surrogate as SU
    return {"workload": "surrogate_8_to_256_trials", "N": 65536, "signals": SG_SIGNALS, "trials_small": 8,
            "trials_equivalent": 256, "max_imf": 10, "sifts_per_imf": 10, "corrected_modes": SU.P_CORR,
            "network": "dilated conv 8 layers x 64 ch, k=3, d=1..128, bf16 / f32 accumulate",
            "weights": weights, "signals_seeds": "30000..30127 (held out)",
            "l2": "flushed between timed steps (256 MiB write)"}


def surrogate_cpu_workload() -> Workload:
    """The plain 256-trial EEMD the surrogate stands in for, as a CPU sample:
    tasks of one held-out 65536-sample signal, the first 2 of 10 IMFs (10
    sifts each), scaled to 100 sifts per task."""
    return Workload("surrogate65k",
                    {"workload": "plain_256_trial_eemd_65536", "N": 65536, "trials": 256, "eps": 0.2,
                     "max_imf": 10, "sifts_per_imf": 10, "storage": "float32", "solve": "float64"},
                    E=256, eps=0.2, max_imf=10, max_sifts=10, tau=0.0, dtype="f32", seed=30000,
                    cpu_tasks=16, cpu_max_imf=2, signals_fn=_surrogate_signal)


def L_times():
    from eemd4cuda_b200 import _lib as L
    return L.KernelTimes()


def run_surrogate(args):
    """One step: the surrogate decomposition of SG_SIGNALS held-out signals of
    65536 samples (8-trial ensemble, network, served modes and gate).  value
    counts the 256 trials the step stands in for."""
    import torch

    rank, local_rank, world = rank_env()
    if world > 1 and rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    from eemd4cuda_b200 import surrogate as SU

    N, S, E_small, E_big = 65536, SG_SIGNALS, 8, 256
    cb = CpuBaseline(surrogate_cpu_workload()) if world == 1 and not args.quick else None

    if SURROGATE_WEIGHTS.exists():
        net = SU.Net(seed=0)
        net.io_increase = SU.load_model(SURROGATE_WEIGHTS, net)
        weights = f"{SURROGATE_WEIGHTS.relative_to(ROOT)}"
    else:
        inp, tgt = SU.generate_pairs(range(10000, 10256), N, E_small, E_big)
        vinp, vtgt = SU.generate_pairs(range(20000, 20032), N, E_small, E_big)
        net, rep = SU.fit(inp, tgt, vinp, vtgt, candidates=2, steps=3000)
        net.io_increase = rep["io_increase"]
        del inp, tgt, vinp, vtgt
        weights = "trained in this run (256 signals, 2 candidates x 3000 steps)"
    xs = SU.make_signals(range(30000, 30000 + S), N)
    sur = SU.SurrogateEEMD(net, S, N, E_small, E_big, SU.engine_params())
    sur.xd.copy_(torch.from_numpy(np.concatenate(xs)))
    flush = torch.empty((2 * L2_BYTES,), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        sur.run(S)
    torch.cuda.synchronize()
    net.check()

    clk = ClockSampler(local_rank)
    clk.start()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sur.run(S)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    clocks = clk.stop()
    ms = total_ms / args.steps
    value = S * N * E_big / (ms / 1e3) / 1e6

    # split: the small ensemble, the network, the stages
    flush.fill_(1)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    sur.imf_sum.zero_()
    sur.mode_count.zero_()
    kt = L_times()
    ev[0].record(stream)
    sur.ens.sums(sur.xd, S, 0, E_small, sur.imf_sum, sur.mode_count, times=kt)
    ev[1].record(stream)
    from eemd4cuda_b200 import _sg as SG
    SG.scale(sur.xd, sur.scale, S, N)
    SG.prepare(sur.imf_sum, sur.mode_count, sur.xd, sur.scale, sur.inp, S, N, sur.K, SU.CH)
    ev[2].record(stream)
    net.infer(sur.inp, sur.out, S, N, sur.chunk, sur.bufs)
    ev[3].record(stream)
    ev[3].synchronize()
    ens_ms, stage_ms, net_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3])
    launches = sum(v["launches"] for v in kt.as_dict().values()) + sur.launches_per_run(S)
    # the step's dominant kernel is the 8-trial ensemble's k_emd: its algorithmic
    # bytes from the knot log of one traced launch (fresh sums, same inputs)
    from eemd4cuda_b200 import _lib as LL
    kt2 = LL.KernelTimes()
    tmp_sum = torch.zeros_like(sur.imf_sum)
    tmp_cnt = torch.zeros_like(sur.mode_count)
    klog = torch.full((S * E_small, sur.K, int(sur.ens.p.max_sifts), 2), -1, dtype=torch.int32, device=dev)
    nmode = torch.zeros((S * E_small,), dtype=torch.int32, device=dev)
    flush.fill_(1)
    LL.run(sur.ens.p, sur.xd, [N] * S, 0, E_small, sur.ens.ws, imf_sum=tmp_sum, mode_count=tmp_cnt, times=kt2,
           knot_log=klog, nmode=nmode)
    torch.cuda.synchronize()
    emd_ev = kt2.as_dict()["emd"]
    emd_bytes = emd_algorithmic_bytes(klog.cpu().numpy(), nmode.cpu().numpy(), [N] * S, E_small, 4)
    emd_gbs = emd_bytes / (emd_ev["ms"] / 1e3) / 1e9 if emd_ev["ms"] > 0 else 0.0
    del tmp_sum, tmp_cnt, klog
    flops = SU.network_flops_per_sample() * S * N
    # bytes of the pass: every layer reads its input and writes its output once (bf16, padded channels)
    net_bytes = sum((lay["cin_p"] + lay["cout_p"]) * 2 for lay in net.layers) * S * N
    hbm_peak, hbm_kind = measured_peak_hbm()
    n_conv = len(SU.DILATIONS) * ((S + sur.chunk - 1) // sur.chunk)
    tflops = flops / (net_ms / 1e3) / 1e12
    peak, peak_kind = measured_peak_bf16()

    # the plain 256-trial EEMD of the same signals, and the errors against it
    g = 16
    ens_plain = SU.Ensembles(g, N, E_big)
    K = sur.K
    ps = torch.empty((g * K * N,), dtype=torch.float64, device=dev)
    pc = torch.empty((g * K,), dtype=torch.int32, device=dev)
    pm = torch.empty((g * K * N,), dtype=torch.float64, device=dev)
    pr = torch.empty((g * N,), dtype=torch.float64, device=dev)
    pn = torch.empty((g,), dtype=torch.int32, device=dev)
    ens_plain.plain(sur.xd[:g * N], g, E_small, ps, pc, pm, pr, pn)  # warm-up
    sur.run(S)
    torch.cuda.synchronize()
    imfs = sur.imfs.cpu().numpy()
    met = sur.metrics.cpu().numpy()
    fb = sur.fallback.cpu().numpy().astype(bool)
    cnt = np.maximum(sur.mode_count.cpu().numpy().reshape(S, K), 1)
    m8 = sur.imf_sum.cpu().numpy().reshape(S, K, N) / cnt[:, :, None]
    plain_ms = 0.0
    e8, es = [], []
    for q0 in range(0, S, g):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens_plain.plain(sur.xd[q0 * N:(q0 + g) * N], g, E_big, ps, pc, pm, pr, pn)
        e1.record(stream)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
        big = pm.cpu().numpy().reshape(g, K, N)
        for j in range(g):
            i = q0 + j
            e8.append([SU.rel_l2(m8[i][k], big[j][k]) for k in range(K)])
            es.append([SU.rel_l2(imfs[i][k], big[j][k]) for k in range(K)])
    e8, es = np.median(np.array(e8), axis=0), np.median(np.array(es), axis=0)

    # end to end through the public call: host signals in, served modes out
    # (fallback signals included)
    served = sur.decompose(xs)
    torch.cuda.synchronize()
    e2e_ms = []
    for _ in range(max(1, min(args.steps, 2))):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        served = sur.decompose(xs)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = statistics.median(e2e_ms)
    nf = sum(st["fallback"] for _, _, st in served)

    cpu = None
    if cb is not None:
        cb.step()
        cpu = cb.describe(cb.value(cb.step(), 100.0))  # 10 IMFs x 10 sifts per task
        cpu["sample"] += "; 256-trial EEMD units (the surrogate's output stands in for them)"
        cb.close()

    line = {
        "metric": SURROGATE_METRIC, "value": round(value, 3),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32+f64",
        "data": "synthetic",
        "config": surrogate_config(weights),
        "speedup_vs_plain_256": round(plain_ms / ms, 2), "plain_256_ms": round(plain_ms, 3),
        "split_ms": {"ensemble_8": round(ens_ms, 3), "prepare": round(stage_ms, 3), "network": round(net_ms, 3)},
        "median_rel_l2_per_imf": {"surrogate": [round(float(v), 4) for v in es],
                                  "ensemble_8": [round(float(v), 4) for v in e8]},
        "gate": {"recon_bound": SU.RECON_BOUND, "io_bound": round(sur.io_bound, 4),
                 "io_form": "increase of |IO| over the 8-trial modes (calibrated, >= 0.05)",
                 "fallbacks": int(fb.sum()), "fallbacks_absolute_io": int((np.abs(met[:, 1]) > SU.IO_BOUND).sum()),
                 "max_recon": float(met[:, 0].max()), "median_abs_io": float(np.median(np.abs(met[:, 1]))),
                 "median_abs_io_8": float(np.median(np.abs(met[:, 3]))),
                 "median_abs_io_all": float(np.median(np.abs(met[:, 2])))},
        "e2e": {"value": round(S * N * E_big / (e2e / 1e3) / 1e6, 3), "unit": UNIT, "ms_per_step": round(e2e, 3),
                "h2d_bytes_per_step": S * N * 4, "d2h_bytes_per_step": S * (K + 1) * N * 8 + S * 3 * 8 + S * 4,
                "fallbacks": nf},
        "gpu_launches": launches * args.steps,
        # the dominant kernel of the step: the 8-trial ensemble
        "roofline": {"bound": "hbm", "kernel": "k_emd (8-trial ensemble)", "achieved": round(emd_gbs, 2),
                     "peak": hbm_peak, "peak_kind": hbm_kind, "unit": "GB/s", "frac": round(emd_gbs / hbm_peak, 4),
                     "traffic": None, "algorithmic_bytes_per_launch": round(emd_bytes),
                     "avg_launch_ms": round(emd_ev["ms"], 4)},
        "roofline_tensor": {"bound": "tensor", "kernel": CONV_KERNEL_NAMES.get(net.conv_kernel, "conv"),
                     "achieved": round(tflops, 2), "peak": peak,
                     "peak_kind": peak_kind, "unit": "TFLOP/s", "frac": round(tflops * 1e12 / (peak * 1e12), 4),
                     "traffic": None, "algorithmic_flops_per_launch": round(flops / n_conv),
                     "avg_launch_ms": round(net_ms / n_conv, 5)},
        # one 64-channel layer does 96 FLOP per byte, below the ridge: the layer's own bound is HBM
        "roofline_hbm": {"bound": "hbm", "kernel": CONV_KERNEL_NAMES.get(net.conv_kernel, "conv"),
                         "achieved": round(net_bytes / (net_ms / 1e3) / 1e9, 2),
                         "peak": hbm_peak, "peak_kind": hbm_kind, "unit": "GB/s",
                         "frac": round(net_bytes / (net_ms / 1e3) / 1e9 / hbm_peak, 4),
                         "algorithmic_bytes_per_pass": net_bytes},
        "clocks": clocks,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# CEEMDAN (emd_ref.py:220-259 semantics) on the engine
# ---------------------------------------------------------------------------
CEEMDAN_WL = Workload(
    "ceemdan48k",
    {"workload": "harmonic_clicks_48k_ceemdan", "N": 48000, "trials": 100, "eps": 0.2, "tau": 0.25,
     "max_sifts": 50, "storage": "float64", "solve": "float64 (seam windows)",
     "noise": "W [E,N] drawn on the device (eemd_philox_normals, seed 0)",
     "signals": 1},
    E=100, eps=0.2, max_imf=1, max_sifts=50, tau=0.25, dtype="f64", seed=1, cpu_tasks=16,
    signals_fn=_harmonic)


def run_ceemdan(args):
    """One step: the whole CEEMDAN of the 48 kHz harmonic signal (stage 0
    noise EMDs plus every stage).  value counts N samples per (stage, trial),
    stage 0 included."""
    import torch

    rank, local_rank, world = rank_env()
    if world > 1 and rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    from eemd4cuda_b200 import _lib as L
    from eemd4cuda_b200 import emd_par as M
    from eemd4cuda_b200.ceemdan import ceemdan

    wl = CEEMDAN_WL
    cb = CpuBaseline(wl) if world == 1 and not args.quick else None
    x = wl.signals()[0]
    N, E = len(x), wl.E
    kw = dict(E=E, eps=wl.eps, seed=0, tau=wl.tau, max_sifts=wl.max_sifts, noise="philox")
    for _ in range(args.warmup):
        c, r, st = ceemdan(x, **kw)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    clk = ClockSampler(local_rank)
    clk.start()
    total = 0.0
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c, r, st = ceemdan(x, **kw)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    clocks = clk.stop()
    ms = total / args.steps
    stages = st["n_imfs"] + 1
    value = N * E * stages / (ms / 1e3) / 1e6
    # the same call with the reference's numpy noise draw (host PCG64, the parity mode)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _, _, st_ref = ceemdan(x, **dict(kw, noise="reference"))
    e1.record(stream)
    e1.synchronize()
    ref_noise_ms = e0.elapsed_time(e1)

    # roofline of k_emd on one stage-1 launch (first IMF of x + beta W[e])
    dev = torch.device("cuda", local_rank)
    p1 = M.make_params(dtype=np.float64, noise_mode=L.EEMD_NOISE_SCALED, eps=float(wl.eps * np.std(x)),
                       tau=wl.tau, max_sifts=wl.max_sifts, max_imf=1, min_extrema=4)
    ws = torch.empty((L.workspace_size(p1, [N], E, False),), dtype=torch.uint8, device=dev)
    Wd = torch.from_numpy(np.random.default_rng(0).standard_normal((E, N))).to(dev)
    xd = torch.from_numpy(x).to(dev)
    imf_sum = torch.zeros((N,), dtype=torch.float64, device=dev)
    cnt = torch.zeros((1,), dtype=torch.int32, device=dev)
    klog = torch.full((E, 1, wl.max_sifts, 2), -1, dtype=torch.int32, device=dev)
    nmode = torch.zeros((E,), dtype=torch.int32, device=dev)
    times = L.KernelTimes()
    L.run(p1, xd, [N], 0, E, ws, noise=Wd, imf_sum=imf_sum, mode_count=cnt)
    L.run(p1, xd, [N], 0, E, ws, noise=Wd, imf_sum=imf_sum, mode_count=cnt, times=times, knot_log=klog,
          nmode=nmode)
    torch.cuda.synchronize()
    kt = times.as_dict()
    ev = kt["emd"]
    emd_bytes = emd_algorithmic_bytes(klog.cpu().numpy(), nmode.cpu().numpy(), [N], E, 8)
    gbs = emd_bytes / (ev["ms"] / 1e3) / 1e9 if ev["ms"] > 0 else 0.0
    peak, peak_kind = measured_peak_hbm()
    launches_stage = sum(v["launches"] for v in kt.values())

    cpu = None
    if cb is not None:
        cb.step()
        cpu = cb.describe(cb.value(cb.step()))
        cpu["sample"] += "; stage-1 tasks (first IMF of x + eps*std(x)*w), the unit of this line"
        cb.close()
    line = {
        "metric": CEEMDAN_METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(wl.config, stages=stages, parallelism="replicas1",
                       note="host numpy computes beta = eps*std(r) and the stop tests between stages, as the "
                            "reference does; value and e2e are the same call (host signal in, host modes out)"),
        "e2e": {"value": round(value, 3), "unit": UNIT, "ms_per_step": round(ms, 3),
                "h2d_bytes_per_step": (E * N + N) * 8, "d2h_bytes_per_step": (2 * stages * N + E) * 8},
        "gpu_launches": (launches_stage * stages + 1) * args.steps,
        "roofline": {"bound": "hbm", "kernel": "k_emd", "stage": 1, "achieved": round(gbs, 2), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(gbs / peak, 4), "traffic": None,
                     "algorithmic_bytes_per_launch": round(emd_bytes), "avg_launch_ms": round(ev["ms"], 5)},
        "noise_modes": sorted(set(st["noise_modes"])), "clocks": clocks,
        "reference_noise": {"ms_per_step": round(ref_noise_ms, 3), "stages": st_ref["n_imfs"] + 1,
                            "note": "W from numpy default_rng(seed) on the host, as the reference draws it"},
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the IMF spectra stage (spectra.py:18-58 semantics) on the device
# ---------------------------------------------------------------------------
SMEM_FFT_MAX = 4096  # longest row libeemd_spectra.so transforms in one shared-memory launch
# eemd_sg_conv's tensor_cores argument -> the kernel it runs
CONV_KERNEL_NAMES = {1: "k_conv_tc", 2: "k_conv_tc2", 3: "k_conv_tma", 4: "k_conv_ws"}


def _fft_radices(m: int):
    """(factors, fully factored) of m over 4, 2 and the odd primes up to 31."""
    k = 0
    for q in (4, 2, *range(3, 32, 2)):
        while m % q == 0:
            m //= q
            k += 1
    return k, m == 1


def fft4_split(n: int):
    """The four-step split (N1, N2) libeemd_spectra.so uses for a length above
    4096: N1 the divisor nearest below sqrt(n) with both factors direct
    lengths up to 4096; None when there is none."""
    if n <= SMEM_FFT_MAX or n > SMEM_FFT_MAX * SMEM_FFT_MAX:
        return None
    n1 = 1
    while (n1 + 1) * (n1 + 1) <= n:
        n1 += 1
    for d in range(n1, 1, -1):
        if n % d:
            continue
        if n // d > SMEM_FFT_MAX:
            break
        if _fft_radices(d)[1] and _fft_radices(n // d)[1]:
            return d, n // d
    return None


def fft_passes(n: int) -> int:
    """Kernel launches of one FFT of length n in libeemd_spectra.so: one
    shared-memory launch up to 4096, two for the four-step split above it,
    else one Stockham pass per factor (4s, 2s, odd primes up to 31); a length
    with a larger prime factor runs Bluestein's 2 + 3 power-of-two transforms
    + 2."""
    k, direct = _fft_radices(n)
    if direct:
        if n <= SMEM_FFT_MAX:
            return 1
        return 2 if fft4_split(n) else max(k, 1)
    L = 1
    while L < 2 * n - 1:
        L <<= 1
    return 4 + 3 * fft_passes(L)


def spectra_launches(n: int, nperseg: int) -> int:
    """Launches of the spectra step: two STFT calls (one launch each when the
    frames are direct lengths up to 4096, else k_frames, the frame FFT and
    k_stft_out) and one Hilbert call (two four-step transforms with the real
    input and the analytic weights in their loads, then k_if_amp; else
    k_promote, FFT, k_analytic, inverse FFT, k_if_amp)."""
    stft = 1 if nperseg <= SMEM_FFT_MAX and _fft_radices(nperseg)[1] else 2 + fft_passes(nperseg)
    hilbert = 5 if _fft_radices(n)[1] and fft4_split(n) else 3 + 2 * fft_passes(n)
    return 2 * stft + hilbert


def run_spectra(args):
    """One step: the Tier-2 spectra of the bench workload's decomposition --
    STFT (nperseg 4096, 50 % overlap) of x and of its 8 ensemble-mean IMFs and
    the Hilbert frequency / amplitude of every IMF -- on device-resident rows.
    value = rows x N / step time."""
    import torch

    rank, local_rank, world = rank_env()
    if world > 1 and rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    from eemd4cuda_b200 import emd_par as M
    from eemd4cuda_b200 import spectra
    from oracle import spectra_oracle as SPO

    wl = WORKLOADS["harmonic48k"]
    x = wl.signals()[0]
    r = M.decompose(x.astype(np.float32), E=wl.E, eps=wl.eps, tau=wl.tau, max_sifts=wl.max_sifts,
                    max_imf=wl.max_imf, seed=wl.seed, dtype=np.float32)
    sr, N, nper = 48000, len(x), 4096
    imfs = torch.from_numpy(np.ascontiguousarray(r.imfs)).to(dev)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(dev).reshape(1, -1)
    rows = 1 + r.n_modes

    def step():
        spectra.stft_device(xd, sr, nper)
        spectra.stft_device(imfs, sr, nper)
        return spectra.hilbert_if_device(imfs, sr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    flush = torch.empty((2 * L2_BYTES,), dtype=torch.uint8, device=dev)
    clk = ClockSampler(local_rank)
    clk.start()
    total = 0.0
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    clocks = clk.stop()
    ms = total / args.steps
    value = rows * N / (ms / 1e3) / 1e6
    # Hilbert alone on the IMFs: algorithmic bytes = read the row, write frequency and amplitude
    flush.fill_(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    spectra.hilbert_if_device(imfs, sr)
    e1.record(stream)
    e1.synchronize()
    h_ms = e0.elapsed_time(e1)
    h_bytes = r.n_modes * N * (8 + 16)
    gbs = h_bytes / (h_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    # end to end through the host API (host rows in, host spectra out)
    hx, himfs = np.ascontiguousarray(x, dtype=np.float64), np.ascontiguousarray(r.imfs)

    def e2e_call():
        spectra.stft_block(hx, sr, nper)
        spectra.stft_block(himfs, sr, nper)
        spectra.hilbert_if(himfs, sr)

    # one untimed call first: it brings the pinned host blocks of the results'
    # sizes into torch's host allocator cache, as the EEMD lines' warm-up does
    e2e_call()
    e2e_ms = []
    for _ in range(max(3, args.steps)):  # the median of at least 3 calls
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_call()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = statistics.median(e2e_ms)
    F, T = nper // 2 + 1, (N + nper - nper // 2) // (nper // 2)
    # CPU: the oracle's numpy restatement of the reference's scipy calls, one core
    t0 = time.perf_counter()
    SPO.stft(hx, sr, nper)
    for k in range(r.n_modes):
        SPO.stft(himfs[k], sr, nper)
        SPO.hilbert_if(himfs[k], sr)
    cpu_s = time.perf_counter() - t0
    line = {
        "metric": "IMF spectra Msamples/s", "value": round(value, 3), "unit": "Msamples/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "spectra_of_harmonic48k_decomposition", "N": N, "rows": rows,
                   "imfs": r.n_modes, "nperseg": nper, "noverlap": nper // 2, "sr": sr,
                   "l2": "flushed between timed steps (256 MiB write)"},
        "e2e": {"value": round(rows * N / (e2e / 1e3) / 1e6, 3), "unit": "Msamples/s", "ms_per_step": round(e2e, 3),
                "h2d_bytes_per_step": rows * N * 8 + r.n_modes * N * 8,
                "d2h_bytes_per_step": rows * F * T * 16 + 2 * r.n_modes * N * 8},
        "gpu_launches": spectra_launches(N, nper) * args.steps,
        "roofline": {"bound": "hbm", "kernel": "hilbert stage (four-step FFT with the real input in its loads, "
                                               "inverse four-step FFT with the analytic weights, k_if_amp)",
                     "achieved": round(gbs, 2), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(gbs / peak, 4), "traffic": None, "algorithmic_bytes": h_bytes,
                     "ms": round(h_ms, 4)},
        "cpu_baseline": {"value": round(rows * N / cpu_s / 1e6, 4), "unit": "Msamples/s", "cores": 1,
                         "kind": "port", "sample": "the whole step once with the oracle's numpy restatement "
                                                    "(numpy FFT, one thread)"},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["surrogate", "ceemdan48k", "spectra48k"],
                    default="harmonic48k")
    ap.add_argument("--quick", action="store_true",
                    help="a brief line: no CPU baseline, no oracle comparison, 3 end-to-end calls")
    ap.add_argument("--no-companions", action="store_true",
                    help="leave out the brief lines of the other workloads from the headline line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "spectra48k":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "spectra48k analyses the engine's IMFs of the "
                              "bench workload (a GPU result); its line carries the numpy restatement's CPU time"}))
            return 0
        return run_spectra(args)
    if args.workload == "ceemdan48k":
        if args.impl == "reference":
            return run_reference(args, CEEMDAN_WL, metric=CEEMDAN_METRIC)
        return run_ceemdan(args)
    if args.workload == "surrogate":
        if args.impl == "reference":
            w = (f"{SURROGATE_WEIGHTS.relative_to(ROOT)}" if SURROGATE_WEIGHTS.exists()
                 else "trained in this run (256 signals, 2 candidates x 3000 steps)")
            return run_reference(args, surrogate_cpu_workload(), metric=SURROGATE_METRIC,
                                 config=surrogate_config(w))
        return run_surrogate(args)
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, wl)
    return run_ours(args, wl)


if __name__ == "__main__":
    sys.exit(main())
