"""Threads per trial and block size, tuned per signal-length bucket and task count.

The engine spreads one (signal, trial) task over a thread-block cluster of C
CTAs of W warps (C x W x 32 threads per trial; W = 4 or 5; float32 storage
runs four or three CTAs per SM, float64 three).  The best (C, W) depends on the signal length (how much work
one CTA's segment holds) and on how many tasks share the launch (how many of
the B200's CTA slots each task can have).  `tune()` measures the persistent
kernel for every (length bucket, task count, W, C) on synthetic signals of
the 48 kHz benchmark kind and writes the fastest (C, W) per (bucket, task
count) to a JSON table (eemd4cuda_b200/tuning/b200_<dtype>.json, committed
with the package); `launch_shape()` looks a launch up in it, and the Python
entry points (`emd_par.decompose`, `decompose_many`) pass the result to the
engine when the caller leaves `EngineConfig.cluster_size` and `cta_warps` at
0.  Without a table entry the engine's own rule applies (eemd_engine.cu
autotune_csize, 4-warp CTAs).  The fast solve's rows per lane is a
build-time constant chosen by measurement.

    python -m eemd4cuda_b200.autotune --dtype f32 [--quick]
"""
from __future__ import annotations

import argparse
import json
import math
import time
from functools import lru_cache
from pathlib import Path

import numpy as np

TABLE_DIR = Path(__file__).resolve().parent / "tuning"
# 49152: about a second of 48 kHz audio, the audio stage's usual segment
BUCKETS = (4096, 8192, 16384, 32768, 49152, 65536, 262144, 1 << 20, 1 << 22)
TASKS = (1, 8, 32, 64, 100, 256, 1024, 4096)
CANDIDATES = (1, 2, 3, 4, 5, 6, 8, 12, 16)   # CTAs per task
WARPS = (4, 5)                                # warps per CTA
MAX_SAMPLES = 1 << 29  # tasks x length per measurement (workspace and time bound)


def table_path(dtype: str) -> Path:
    return TABLE_DIR / f"b200_{dtype}.json"


@lru_cache(maxsize=4)
def _table(dtype: str):
    p = table_path(dtype)
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return [(int(e["n"]), int(e["tasks"]), int(e["cluster_size"]), int(e.get("cta_warps", 4)))
            for e in d["entries"]]


def launch_shape(n_ref: int, n_tasks: int, dtype: str, n_min: int | None = None) -> tuple:
    """Tuned (CTAs per task, warps per CTA) for a launch of n_tasks tasks
    whose signals have a median length of n_ref samples and a shortest one
    of n_min (default n_ref): the nearest entry in log length, then in log
    task count, with no more CTAs than give the shortest signal 2048 samples
    each; (0, 0) when the table has no entry for that storage type."""
    tab = _table(dtype)
    if not tab:
        return 0, 0
    n_min = n_ref if n_min is None else n_min
    key = (id(tab), int(n_ref), int(n_tasks), int(n_min))
    hit = _SHAPES.get(key)
    if hit is not None:
        return hit
    lengths = sorted({n for n, _, _, _ in tab})
    bn = min(lengths, key=lambda n: abs(math.log(n) - math.log(max(n_ref, 1))))
    rows = [(t, c, w) for n, t, c, w in tab if n == bn]
    t, c, w = min(rows, key=lambda r: abs(math.log(r[0]) - math.log(max(n_tasks, 1))))
    # a cluster needs at least 2048 samples per CTA (the engine's own bound)
    while c > 1 and n_min // c < 2048:
        c -= 1
    if len(_SHAPES) > 4096:
        _SHAPES.clear()
    _SHAPES[key] = (c, w)
    return c, w


_SHAPES: dict = {}  # looked-up shapes per (table, lengths, task count)


def cluster_size(n_min: int, n_tasks: int, dtype: str) -> int:
    """The CTAs-per-task half of launch_shape()."""
    return launch_shape(n_min, n_tasks, dtype)[0]


def _measure(n: int, tasks: int, dtype: str, c: int, reps: int, nw: int = 4) -> float:
    """ms of the persistent kernel for `tasks` trials of one n-sample signal
    (2 IMFs x 5 fixed sifts, Philox noise) with clusters of c CTAs of nw warps."""
    import torch

    from . import _lib as L
    from . import emd_par as M
    from . import signals

    dt = np.float32 if dtype == "f32" else np.float64
    x = signals.harmonic_clicks(n, seed=1).astype(dt)
    p = M.make_params(dtype=dt, noise_mode=L.EEMD_NOISE_PHILOX, eps=0.2, seed=1, tau=0.0, max_sifts=5,
                      max_imf=2, config=M.EngineConfig(cluster_size=c, cta_warps=nw))
    dev = torch.device("cuda", torch.cuda.current_device())
    xd = torch.from_numpy(x).to(dev)
    ws = torch.empty((L.workspace_size(p, [n], tasks, False),), dtype=torch.uint8, device=dev)
    best = float("inf")
    for r in range(reps + 1):
        t = L.KernelTimes()
        L.run(p, xd, [n], 0, tasks, ws, times=t)
        if r:
            best = min(best, t.as_dict()["emd"]["ms"])
    del ws
    return best


def tune(dtype: str = "f32", quick: bool = False, reps: int = 2, buckets=None) -> dict:
    import torch

    buckets = tuple(buckets) if buckets else (BUCKETS[:4] if quick else BUCKETS)
    entries = []
    for n in buckets:
        for tasks in TASKS:
            if n * tasks > MAX_SAMPLES or (dtype == "f64" and n * tasks > MAX_SAMPLES // 2):
                continue
            times = {}
            for nw in WARPS:
                for c in CANDIDATES:
                    if n // c < 2048 and c > 1:
                        continue
                    try:
                        times[(nw, c)] = _measure(n, tasks, dtype, c, reps, nw)
                    except Exception as e:  # a cluster size the device cannot launch
                        times[(nw, c)] = None
                        print(f"n={n} tasks={tasks} W={nw} C={c}: {e}", flush=True)
                    torch.cuda.empty_cache()
            ok = {k: t for k, t in times.items() if t is not None}
            bw, bc = min(ok, key=ok.get)
            entries.append({"n": n, "tasks": tasks, "cluster_size": bc, "cta_warps": bw,
                            "ms": {f"{w}x{c}": (round(t, 4) if t is not None else None)
                                   for (w, c), t in times.items()}})
            print(json.dumps(entries[-1]), flush=True)
    return {"device": torch.cuda.get_device_name(), "dtype": dtype,
            "workload": "harmonic + pink noise + clicks (48 kHz kind), Philox noise 0.2 std, 2 IMFs x 5 fixed sifts",
            "measured": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), "entries": entries}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=None)
    ap.add_argument("--buckets", default="", help="comma-separated lengths to measure (default: all buckets)")
    ap.add_argument("--merge", default="", help="a table whose entries for other lengths are kept")
    a = ap.parse_args()
    d = tune(a.dtype, a.quick, buckets=[int(v) for v in a.buckets.split(",") if v])
    if a.merge:
        old = json.loads(Path(a.merge).read_text())
        mine = {e["n"] for e in d["entries"]}
        d["entries"] = sorted([e for e in old["entries"] if e["n"] not in mine] + d["entries"],
                              key=lambda e: (e["n"], e["tasks"]))
        d["measured"] = f'{old.get("measured")}; lengths {sorted(mine)}: {d["measured"]}'
    out = Path(a.out) if a.out else table_path(a.dtype)
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text(json.dumps(d, indent=1))
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
