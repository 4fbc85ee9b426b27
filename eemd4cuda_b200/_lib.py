"""ctypes binding of libeemd_b200.so (the C ABI declared in include/eemd_b200.h).

The library is the product: there is no CPU fallback.  Loading fails loudly
when the shared object is missing or was built for a different ABI.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int32, c_int64, c_size_t, c_uint64, c_void_p
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_DIR = _PKG / "lib"

EEMD_OK = 0
EEMD_E_BADARG = -1
EEMD_E_NOMEM = -2
EEMD_E_KNOT_OVERFLOW = -3
EEMD_E_TIMEOUT = -4
EEMD_E_CUDA = -5
EEMD_E_NOTSUP = -6
EEMD_E_STATIC_CAPACITY = -7
STATIC_SCRATCH_BYTES = 64 * 1024 * 1024

EEMD_F64 = 0
EEMD_F32 = 1
EEMD_END_NATURAL = 0
EEMD_END_MIRROR = 1
EEMD_RULES_REF = 0
EEMD_RULES_NUMBA = 1
EEMD_NOISE_NONE = 0
EEMD_NOISE_PHILOX = 1
EEMD_NOISE_INJECTED = 2
EEMD_NOISE_PREPERTURBED = 3
EEMD_NOISE_SCALED = 4
ABI_VERSION = 2

# every symbol include/eemd_b200.h declares
EXPORTS = ("eemd_default_params", "eemd_version", "eemd_strerror",
           "eemd_workspace_size", "eemd_run", "eemd_run_traced", "eemd_run_static",
           "eemd_finalize", "eemd_philox_normals")

KERNEL_KINDS = ("sigma", "emd", "reduce", "outputs", "k4", "k5", "k6", "k7")


class EemdParams(ctypes.Structure):
    """Mirror of `eemd_params` (include/eemd_b200.h)."""

    _fields_ = [
        ("dtype", c_int32),
        ("noise_mode", c_int32),
        ("eps", c_double),
        ("seed", c_uint64),
        ("tau", c_double),
        ("max_sifts", c_int32),
        ("max_imf", c_int32),
        ("min_extrema", c_int32),
        ("end_mode", c_int32),
        ("rules", c_int32),
        ("exact", c_int32),
        ("tile", c_int32),
        ("knots_per_block", c_int32),
        ("halo", c_int32),
        ("watchdog", c_int64),
        ("cluster_size", c_int32),
        ("reserved", c_int32),
        ("cta_warps", c_int32),
        ("reserved2", c_int32),
    ]


class KernelTimes(ctypes.Structure):
    """Mirror of `eemd_kernel_times`."""

    _fields_ = [("ms", c_double * 8), ("launches", c_int64 * 8)]

    def as_dict(self) -> dict:
        return {k: {"ms": float(self.ms[i]), "launches": int(self.launches[i])}
                for i, k in enumerate(KERNEL_KINDS) if not k.startswith("k")}


class EngineError(RuntimeError):
    """A non-zero status from the engine."""

    def __init__(self, status: int, where: str = ""):
        self.status = int(status)
        super().__init__(f"{where}: {strerror(status)} (status {status})")


_LIB = None


def lib_path() -> Path:
    """Path of the engine library (EEMD_B200_LIB overrides, e.g. the checked build)."""
    env = os.environ.get("EEMD_B200_LIB")
    if env:
        return Path(env)
    return LIB_DIR / "libeemd_b200.so"


def load() -> ctypes.CDLL:
    """Load (once) and type the engine library; raise if it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    _LIB = load_variant(lib_path())
    return _LIB


def load_variant(path) -> ctypes.CDLL:
    """Load and type a build of the engine library at `path` (for example the
    bounds-checked build) next to the default one; raise if it is absent."""
    path = Path(path)
    if not path.exists():
        raise RuntimeError(
            f"EEMD engine library not found at {path}; build it with "
            "`python -m eemd4cuda_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(path))
    for name in EXPORTS:
        if not hasattr(lib, name):
            raise RuntimeError(f"{path} does not export {name}")
    lib.eemd_default_params.argtypes = [POINTER(EemdParams)]
    lib.eemd_default_params.restype = None
    lib.eemd_version.argtypes = []
    lib.eemd_version.restype = c_int32
    lib.eemd_strerror.argtypes = [c_int32]
    lib.eemd_strerror.restype = ctypes.c_char_p
    lib.eemd_workspace_size.argtypes = [POINTER(EemdParams), POINTER(c_int64), c_int32, c_int32,
                                        c_int32, POINTER(c_size_t)]
    lib.eemd_workspace_size.restype = c_int32
    lib.eemd_run.argtypes = [
        POINTER(EemdParams), c_void_p, POINTER(c_int64), c_int32, c_int32, c_int32,
        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
        c_void_p, c_size_t, c_void_p]
    lib.eemd_run.restype = c_int32
    lib.eemd_run_traced.argtypes = lib.eemd_run.argtypes + [POINTER(KernelTimes)]
    lib.eemd_run_traced.restype = c_int32
    lib.eemd_run_static.argtypes = lib.eemd_run.argtypes[:16] + [c_void_p]
    lib.eemd_run_static.restype = c_int32
    lib.eemd_finalize.argtypes = [POINTER(EemdParams), c_void_p, POINTER(c_int64), c_int32,
                                  c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.eemd_finalize.restype = c_int32
    lib.eemd_philox_normals.argtypes = [ctypes.c_uint64, c_int32, c_int32, c_int32, c_int64, c_void_p, c_void_p]
    lib.eemd_philox_normals.restype = c_int32
    v = lib.eemd_version()
    if v != ABI_VERSION:
        raise RuntimeError(f"{path}: ABI version {v}, expected {ABI_VERSION}")
    return lib


def strerror(status: int) -> str:
    try:
        return load().eemd_strerror(int(status)).decode()
    except Exception:  # library not loadable: still describe the code
        return {0: "ok", -1: "invalid argument", -2: "workspace too small",
                -3: "knot buffer capacity exceeded", -4: "device wait gave up (watchdog)",
                -5: "CUDA runtime error", -6: "unsupported parameter combination",
                -7: "problem needs more scratch than the static scratch of eemd_run_static"}.get(
                    int(status), "unknown status")


def check(status: int, where: str) -> None:
    if status == EEMD_E_BADARG:
        raise ValueError(f"{where}: {strerror(status)}")
    if status != EEMD_OK:
        raise EngineError(status, where)


def default_params() -> EemdParams:
    p = EemdParams()
    load().eemd_default_params(ctypes.byref(p))
    return p


def lengths_array(lengths) -> ctypes.Array:
    arr = (c_int64 * len(lengths))()
    for i, n in enumerate(lengths):
        arr[i] = int(n)
    return arr


def workspace_size(p: EemdParams, lengths, trial_count: int, imfs_external: bool) -> int:
    out = c_size_t(0)
    la = lengths_array(lengths)
    check(load().eemd_workspace_size(ctypes.byref(p), la, len(lengths), int(trial_count),
                                     int(bool(imfs_external)), ctypes.byref(out)),
          "eemd_workspace_size")
    return int(out.value)


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


def run(p: EemdParams, x, lengths, trial_begin: int, trial_count: int, ws, *, noise=None,
        imfs=None, resid_out=None, imf_sum=None, mode_count=None, nsift=None, nmode=None,
        mode_sifts=None, knot_log=None, flags=None, stream=None, times: KernelTimes | None = None,
        ws_bytes: int | None = None, lib: ctypes.CDLL | None = None) -> None:
    """eemd_run on torch device tensors (all optional outputs may be None).
    With `times`, runs eemd_run_traced and fills per-kernel event timings.
    `lib`: another build of the library (load_variant) instead of the default."""
    import torch

    la = lengths_array(lengths)
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    nb = ws.numel() * ws.element_size() if ws_bytes is None else int(ws_bytes)
    args = (ctypes.byref(p), _ptr(x), la, len(lengths), int(trial_begin),
            int(trial_count), _ptr(noise), _ptr(imfs), _ptr(resid_out), _ptr(imf_sum),
            _ptr(mode_count), _ptr(nsift), _ptr(nmode), _ptr(mode_sifts),
            _ptr(knot_log), _ptr(flags), _ptr(ws), nb, c_void_p(st))
    lib = lib or load()
    if times is None:
        rc = lib.eemd_run(*args)
    else:
        rc = lib.eemd_run_traced(*args, ctypes.byref(times))
    check(rc, "eemd_run")


def run_static(p: EemdParams, x, lengths, trial_begin: int, trial_count: int, *, noise=None,
               imfs=None, resid_out=None, imf_sum=None, mode_count=None, nsift=None, nmode=None,
               mode_sifts=None, knot_log=None, flags=None, stream=None) -> None:
    """eemd_run_static: the engine on the library's own static device scratch,
    for callers that must not allocate device memory (no workspace argument)."""
    import torch

    la = lengths_array(lengths)
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = load().eemd_run_static(ctypes.byref(p), _ptr(x), la, len(lengths), int(trial_begin),
                                int(trial_count), _ptr(noise), _ptr(imfs), _ptr(resid_out),
                                _ptr(imf_sum), _ptr(mode_count), _ptr(nsift), _ptr(nmode),
                                _ptr(mode_sifts), _ptr(knot_log), _ptr(flags), c_void_p(st))
    check(rc, "eemd_run_static")


def philox_normals(seed: int, signal: int, trial_begin: int, trial_count: int, n: int, out,
                   stream=None) -> None:
    """eemd_philox_normals into a float64 device tensor out [trial_count * n]."""
    import torch

    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = load().eemd_philox_normals(int(seed) & 0xFFFFFFFFFFFFFFFF, int(signal), int(trial_begin),
                                    int(trial_count), int(n), _ptr(out), c_void_p(st))
    check(rc, "eemd_philox_normals")


def finalize(p: EemdParams, x, lengths, imf_sum, mode_count, imf_mean, residual, n_modes,
             stream=None) -> None:
    import torch

    la = lengths_array(lengths)
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = load().eemd_finalize(ctypes.byref(p), _ptr(x), la, len(lengths), _ptr(imf_sum),
                              _ptr(mode_count), _ptr(imf_mean), _ptr(residual), _ptr(n_modes),
                              c_void_p(st))
    check(rc, "eemd_finalize")
