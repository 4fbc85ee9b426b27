"""ctypes binding of libeemd_surrogate.so (the C ABI of include/eemd_surrogate.h)."""
from __future__ import annotations

import ctypes
from ctypes import c_float, c_int32, c_int64, c_void_p
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
SG_OK = 0
SG_E_BADARG = -1
SG_E_TIMEOUT = -4
SG_E_CUDA = -5
ABI_VERSION = 1
EXPORTS = ("eemd_sg_version", "eemd_sg_conv", "eemd_sg_pack", "eemd_sg_wgrad", "eemd_sg_loss", "eemd_sg_adam")

_lib = None


class SurrogateError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: status {status}")
        self.status = status


def lib_path() -> Path:
    return LIB_DIR / "libeemd_surrogate.so"


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        raise RuntimeError(f"{path} is missing: build it with `python -m eemd4cuda_b200.build`")
    lib = ctypes.CDLL(str(path))
    lib.eemd_sg_version.restype = c_int32
    if lib.eemd_sg_version() != ABI_VERSION:
        raise RuntimeError("libeemd_surrogate.so ABI version mismatch")
    lib.eemd_sg_conv.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32,
                                 c_int32, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_int64, c_void_p]
    lib.eemd_sg_pack.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_void_p]
    lib.eemd_sg_wgrad.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32,
                                  c_int32, c_int32, c_int32, c_void_p]
    lib.eemd_sg_loss.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32,
                                 c_int32, c_int32, c_void_p]
    lib.eemd_sg_adam.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_float, c_float, c_float,
                                 c_float, c_int32, c_void_p]
    for f in EXPORTS[1:]:
        getattr(lib, f).restype = c_int32
    _lib = lib
    return lib


def _p(t):
    return c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    import torch
    return c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(rc, where):
    if rc != SG_OK:
        raise SurrogateError(rc, where)


def conv(x, wpk, bias, y, B, T, cin, cout, dil, direction=1, relu=False, mask=None, tensor_cores=True,
         err=None, spin_limit=0):
    _check(load().eemd_sg_conv(_p(x), _p(wpk), _p(bias), _p(y), B, T, cin, cout, dil, direction, int(relu),
                               _p(mask), int(tensor_cores), _p(err), spin_limit, _stream()), "eemd_sg_conv")


def pack(w, wpk, n_rows, c, nv, cv, transpose=False):
    _check(load().eemd_sg_pack(_p(w), _p(wpk), n_rows, c, nv, cv, int(transpose), _stream()), "eemd_sg_pack")


def wgrad(dy, x, dw, db, B, T, n_rows, c, nv, cv, dil):
    _check(load().eemd_sg_wgrad(_p(dy), _p(x), _p(dw), _p(db), B, T, n_rows, c, nv, cv, dil, _stream()),
           "eemd_sg_wgrad")


def loss(out, base, target, dout, acc, B, T, c, cv, margin):
    _check(load().eemd_sg_loss(_p(out), _p(base), _p(target), _p(dout), _p(acc), B, T, c, cv, margin,
                               _stream()), "eemd_sg_loss")


def adam(p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    _check(load().eemd_sg_adam(_p(p), _p(g), _p(m), _p(v), p.numel(), lr, b1, b2, eps, step, _stream()),
           "eemd_sg_adam")
