"""Result files written from device buffers.

Two formats of the reference, byte-compatible in their keys and dtypes:

  * EMDResult.save / load (emd_par.py:84-97): imfs, residual, n_modes and the
    scalar stats; `save_result` writes it from device tensors.
  * imfs.npz (audio_eemd/report.py:177-194): x, t, imfs [n_modes, N],
    residual, n_modes (int64) and stat_<key> for scalar / integer-list stats;
    `write_imfs_npz` takes host arrays or device tensors.

`AsyncWriter` moves device results to pinned host memory on a copy stream,
ordered after the stream that produced them, and writes the file on a host
thread, so the GPU can go on with the next segment while the previous one is
compressed and written.  Nothing here computes on the results.
"""
from __future__ import annotations

import threading
from pathlib import Path

import numpy as np

__all__ = ["imfs_npz_payload", "write_imfs_npz", "save_result", "AsyncWriter"]


def _host(a):
    if hasattr(a, "is_cuda"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def imfs_npz_payload(x, t, imfs, residual, n_modes, stats) -> dict:
    """The arrays of imfs.npz, as report.write_imfs_npz lays them out."""
    payload = {"x": _host(x), "t": _host(t), "imfs": _host(imfs), "residual": _host(residual),
               "n_modes": np.int64(n_modes)}
    for k, v in stats.items():
        if k == "x":
            continue  # the input is stored once, as 'x'
        if isinstance(v, (int, float, bool, np.integer, np.floating, np.bool_)):
            payload[f"stat_{k}"] = np.asarray(v)
        elif isinstance(v, (list, tuple)) and all(isinstance(i, (int, np.integer)) for i in v):
            payload[f"stat_{k}"] = np.asarray(v, dtype=np.int64)
    return payload


def write_imfs_npz(outdir, x, t, imfs, residual, n_modes, stats) -> Path:
    """outdir/imfs.npz (compressed)."""
    p = Path(outdir) / "imfs.npz"
    np.savez_compressed(p, **imfs_npz_payload(x, t, imfs, residual, n_modes, stats))
    return p


def save_result(path, imfs, residual, n_modes, stats=None):
    """EMDResult.save's file from host arrays or device tensors."""
    from .emd_par import EMDResult
    EMDResult(imfs=_host(imfs), residual=_host(residual), n_modes=int(n_modes), stats=dict(stats or {})).save(path)


class AsyncWriter:
    """Device results -> pinned host buffers (copy stream) -> imfs.npz on a host thread.

        w = AsyncWriter()
        w.submit(outdir, x_host, t_host, imf_mean_dev[:n_modes], resid_dev, n_modes, stats)
        ...            # next segment's kernels run meanwhile
        w.close()      # waits for every file

    The device tensors must not be overwritten before their copies end:
    `submit` records an event on the producing stream, the copy stream waits
    for it, and the tensors are handed back only when `wait_copies()` or
    `close()` returns (or use fresh buffers per segment)."""

    def __init__(self):
        import torch
        self.torch = torch
        self.stream = torch.cuda.Stream()
        self.threads: list[threading.Thread] = []
        self.events = []
        self.errors: list[BaseException] = []

    def submit(self, outdir, x, t, imfs, residual, n_modes, stats) -> Path:
        torch = self.torch
        produced = torch.cuda.Event()
        produced.record(torch.cuda.current_stream())
        hosts = []
        with torch.cuda.stream(self.stream):
            self.stream.wait_event(produced)
            for a in (imfs, residual):
                if hasattr(a, "is_cuda") and a.is_cuda:
                    h = torch.empty(a.shape, dtype=a.dtype, pin_memory=True)
                    h.copy_(a, non_blocking=True)
                    a.record_stream(self.stream)
                    hosts.append(h)
                else:
                    hosts.append(a)
            done = torch.cuda.Event()
            done.record(self.stream)
        self.events.append(done)
        path = Path(outdir) / "imfs.npz"

        def write():
            try:
                done.synchronize()
                write_imfs_npz(outdir, x, t, _host(hosts[0]), _host(hosts[1]), n_modes, stats)
            except BaseException as e:  # reported by close()
                self.errors.append(e)

        th = threading.Thread(target=write, daemon=True)
        th.start()
        self.threads.append(th)
        return path

    def wait_copies(self):
        for e in self.events:
            e.synchronize()
        self.events.clear()

    def close(self):
        self.wait_copies()
        for th in self.threads:
            th.join()
        self.threads.clear()
        if self.errors:
            raise self.errors[0]
