#!/usr/bin/env python
"""EEMD throughput on one B200 (or N independent replicas), one JSON line.

Workload (one "step"): full EEMD of 1 s of 48 kHz synthetic audio -- harmonic
tone f0=220 Hz with 8 partials (1/k), pink noise at -30 dB, 5 decaying clicks,
seed 1 -- N=48000 samples, 100 trials, Philox noise 0.2*std(x), 8 IMFs,
fixed 10 sifts per IMF, float32 storage with float64 spline solve.
Metric: Msamples*trials/s = N*E / step time (whole job: summed over ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's CPU algorithm (the numpy port in
oracle/, emd_ref.py semantics, float64) on the host cores with a spawn process
pool, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N = 48000
E = 100
EPS = 0.2
MAX_IMF = 8
MAX_SIFTS = 10
TAU = 0.0          # SD < 0 never holds: every IMF gets exactly MAX_SIFTS sifts
SEED = 1
METRIC = "EEMD Msamples*trials/s"
UNIT = "Msamples*trials/s"
L2_BYTES = 126 * 1024 * 1024
CONFIG = {"workload": "harmonic_clicks_48k_eemd", "N": N, "trials": E, "eps": EPS,
          "max_imf": MAX_IMF, "sifts_per_imf": MAX_SIFTS, "storage": "float32",
          "solve": "float64", "noise": "philox", "signals": 1,
          "l2": "flushed between timed steps (256 MiB write)"}


def rank_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def workload_signal():
    from eemd4cuda_b200 import signals
    return signals.harmonic_clicks(N, seed=SEED)


# ---------------------------------------------------------------------------
# CPU side (reference algorithm, numpy port)
# ---------------------------------------------------------------------------
class CpuBaseline:
    """emd_1d of x + noise_e for a bounded number of trials in a spawn pool."""

    def __init__(self, trials: int | None = None):
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor

        self.cores = os.cpu_count() or 1
        self.trials = trials or max(4, min(self.cores, 32))
        self.x = workload_signal().astype(np.float32).astype(np.float64)
        sigma = EPS * np.std(self.x)
        rng = np.random.default_rng(SEED)
        self.noises = rng.standard_normal((self.trials, N)) * sigma
        self.pool = ProcessPoolExecutor(max_workers=self.cores, mp_context=mp.get_context("spawn"))

    def step(self) -> float:
        from concurrent.futures import as_completed
        from oracle import emd_oracle as O

        kw = dict(tau=TAU, max_sifts=MAX_SIFTS, max_imf=MAX_IMF)
        t0 = time.perf_counter()
        futs = [self.pool.submit(O._trial_worker, (self.x, self.noises[e], kw))
                for e in range(self.trials)]
        for f in as_completed(futs):
            f.result()
        return time.perf_counter() - t0

    def value(self, seconds: float) -> float:
        return self.trials * N / seconds / 1e6

    def describe(self, v: float) -> dict:
        return {"value": round(v, 4), "unit": UNIT, "cores": self.cores, "kind": "port",
                "sample": f"{self.trials} of the {E} trials of the workload (emd_1d, float64, "
                          f"tau=0 / {MAX_SIFTS} sifts, {MAX_IMF} IMFs) in a {self.cores}-process pool"}

    def close(self):
        self.pool.shutdown()


def run_reference(args):
    rank, _, world = rank_env()
    if rank != 0:
        return 0
    cb = CpuBaseline()
    for _ in range(args.warmup):
        cb.step()
    ts = [cb.step() for _ in range(args.steps)]
    cb.close()
    sec = sum(ts) / len(ts)
    v = cb.value(sec)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, storage="float64", sample_trials=cb.trials),
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


def emd_algorithmic_bytes(klog: np.ndarray, nmode: np.ndarray, bytes_el: int) -> float:
    """Algorithmic bytes of one k_emd launch, from the per-sift knot log.

    Per trial: read x and write the residual (2*N*b) and the first knot list
    (P0*(4+b)).  Per sift with P = maxima+minima knots: the solve reads the knots
    (P*(4+b)) and writes the second derivatives (8*P); the sweep reads and writes
    h (2*N*b), reads knots and second derivatives (P*(4+b+8)) and writes the
    next knot list (P'*(4+b)).  The sift that closes an IMF also reads and
    writes the residual (2*N*b)."""
    total = 0.0
    kb = 4 + bytes_el
    for e in range(klog.shape[0]):
        seq = []
        for m in range(int(nmode[e])):
            for k in range(klog.shape[2]):
                a, b = klog[e, m, k]
                if a < 0:
                    break
                seq.append((m, int(a) + int(b)))
        total += 2 * N * bytes_el
        if seq:
            total += seq[0][1] * kb
        for i, (m, P) in enumerate(seq):
            Pn = seq[i + 1][1] if i + 1 < len(seq) else P
            total += P * kb + 8 * P                      # solve
            total += 2 * N * bytes_el + P * (kb + 8) + Pn * kb   # sweep
            if i + 1 == len(seq) or seq[i + 1][0] != m:
                total += 2 * N * bytes_el                # residual update at the IMF close
    return total


def run_ours(args):
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

    from eemd4cuda_b200 import _lib as L
    from eemd4cuda_b200 import emd_par as M

    # the CPU baseline pool is started before any GPU work (spawn context)
    cb = CpuBaseline() if (rank == 0 and world == 1) else None

    x = workload_signal().astype(np.float32)
    p = M.make_params(dtype=np.float32, noise_mode=L.EEMD_NOISE_PHILOX, eps=EPS, seed=SEED + rank,
                      tau=TAU, max_sifts=MAX_SIFTS, max_imf=MAX_IMF)
    xd = torch.from_numpy(x).to(dev)
    ws = torch.empty((L.workspace_size(p, [N], E, False),), dtype=torch.uint8, device=dev)
    imf_sum = torch.zeros((MAX_IMF, N), dtype=torch.float64, device=dev)
    mode_count = torch.zeros((MAX_IMF,), dtype=torch.int32, device=dev)
    imf_mean = torch.empty((MAX_IMF, N), dtype=torch.float64, device=dev)
    resid = torch.empty((N,), dtype=torch.float64, device=dev)
    nmodes = torch.empty((1,), dtype=torch.int32, device=dev)
    flush = torch.empty((2 * L2_BYTES,), dtype=torch.uint8, device=dev)

    def step(times=None, klog=None, nmode=None):
        imf_sum.zero_()
        mode_count.zero_()
        L.run(p, xd, [N], 0, E, ws, imf_sum=imf_sum, mode_count=mode_count, times=times,
              knot_log=klog, nmode=nmode)
        L.finalize(p, xd, [N], imf_sum, mode_count, imf_mean, resid, nmodes)

    for _ in range(args.warmup):
        step()
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
        step()
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
    value = world * N * E / (ms / 1e3) / 1e6

    # ---- per-kernel split (traced step, event pair around every launch) ----
    times = L.KernelTimes()
    klog = torch.full((E, MAX_IMF, MAX_SIFTS, 2), -1, dtype=torch.int32, device=dev)
    nmode = torch.zeros((E,), dtype=torch.int32, device=dev)
    flush.fill_(1)
    step(times=times, klog=klog, nmode=nmode)
    torch.cuda.synchronize()
    kt = times.as_dict()
    launches_per_step = sum(v["launches"] for v in kt.values()) + 1  # + k_finalize
    ev = kt["emd"]
    emd_bytes = emd_algorithmic_bytes(klog.cpu().numpy(), nmode.cpu().numpy(), 4)
    emd_gbs = emd_bytes / (ev["ms"] / 1e3) / 1e9 if ev["ms"] > 0 else 0.0
    peak, peak_kind = measured_peak_hbm()
    traffic = None
    tf = ROOT / "profiles" / "emd_traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get("bytes_per_launch")
        except ValueError:
            traffic = None

    # ---- end to end through the public API (host buffers) ----
    def e2e_call():
        return M.decompose(x, E=E, eps=EPS, tau=TAU, max_sifts=MAX_SIFTS, max_imf=MAX_IMF,
                           seed=SEED + rank, dtype=np.float32)

    for _ in range(args.warmup):
        e2e_call()
    torch.cuda.synchronize()
    e2e_ms = []
    n_modes_e2e = MAX_IMF
    for i in range(max(args.steps, 1)):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = e2e_call()
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        n_modes_e2e = r.n_modes
    e2e = statistics.median(e2e_ms)
    if dist:
        t = torch.tensor([e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())
    e2e_value = world * N * E / (e2e / 1e3) / 1e6

    cpu = None
    if cb is not None:
        cb.step()  # warm the pool's imports
        cs = cb.step()
        cpu = cb.describe(cb.value(cs))
        cb.close()

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": dict(CONFIG, parallelism=f"replicas{world}"),
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "ms_per_step": round(e2e, 4),
                "h2d_bytes_per_step": N * 4,
                "d2h_bytes_per_step": n_modes_e2e * N * 8 + N * 8 + 3 * E * 4},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "kernel": "k_emd", "achieved": round(emd_gbs, 2),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(emd_gbs / peak, 4),
                     "traffic": traffic, "algorithmic_bytes_per_launch":
                         round(emd_bytes / max(ev["launches"], 1)),
                     "avg_launch_ms": round(ev["ms"] / max(ev["launches"], 1), 5)},
        "kernel_split_ms": {k: round(v["ms"], 4) for k, v in kt.items()},
        "kernel_launches": {k: v["launches"] for k, v in kt.items()},
        "clocks": clocks,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
