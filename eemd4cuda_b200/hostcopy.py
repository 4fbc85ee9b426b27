"""Copies of large results out of the pinned staging buffers into fresh arrays.

The first touch of a fresh numpy array page-faults, so one thread fills it
at a few GB/s (a 738 MB result: ~185 ms measured on a 8-core host).  numpy
releases the GIL for plain copies, so slices copied on several threads
spread both the faults and the memcpy (~30 ms with 8 threads on that host).
"""
from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

PARALLEL_BYTES = 16 << 20  # smaller results are copied on the calling thread
WORKERS = max(1, min(8, os.cpu_count() or 1))
_POOL = None
_POOL_LOCK = threading.Lock()


def _pool() -> ThreadPoolExecutor:
    global _POOL
    with _POOL_LOCK:
        if _POOL is None:
            _POOL = ThreadPoolExecutor(max_workers=WORKERS, thread_name_prefix="eemd-copy")
        return _POOL


def prefault(arrays) -> list:
    """Touch every page of fresh arrays on the copy threads (zero-fills 16 MiB
    slices) and return the futures: started before a device computation, the
    page faults happen while the device works instead of during the copies."""
    pool = _pool()
    futs = []
    for a in arrays:
        flat = a.reshape(-1)
        step = max(1, PARALLEL_BYTES // max(a.itemsize, 1))
        futs += [pool.submit(np.copyto, flat[i:i + step], 0) for i in range(0, flat.size, step)]
    return futs


def copy_into(dst: np.ndarray, src: np.ndarray) -> None:
    """dst[...] = src (parallel slices above 16 MiB when both are C-contiguous)."""
    if src.nbytes < PARALLEL_BYTES or not (src.flags.c_contiguous and dst.flags.c_contiguous):
        np.copyto(dst, src)
        return
    s, d = src.reshape(-1), dst.reshape(-1)
    pool = _pool()
    step = -(-s.size // WORKERS)
    futs = [pool.submit(np.copyto, d[i:i + step], s[i:i + step]) for i in range(0, s.size, step)]
    for f in futs:
        f.result()


def fresh_copy(src: np.ndarray) -> np.ndarray:
    """A new C-contiguous array equal to src (parallel slices above 16 MiB)."""
    src = np.asarray(src)
    dst = np.empty(src.shape, dtype=src.dtype)
    if src.nbytes < PARALLEL_BYTES or not src.flags.c_contiguous:
        np.copyto(dst, src)
        return dst
    s, d = src.reshape(-1), dst.reshape(-1)
    pool = _pool()
    step = -(-s.size // WORKERS)
    futs = [pool.submit(np.copyto, d[i:i + step], s[i:i + step]) for i in range(0, s.size, step)]
    for f in futs:
        f.result()
    return dst
