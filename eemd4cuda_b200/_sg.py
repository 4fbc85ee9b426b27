"""ctypes binding of libeemd_surrogate.so (the C ABI of include/eemd_surrogate.h)."""
from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int32, c_int64, c_void_p
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
SG_OK = 0
SG_E_BADARG = -1
SG_E_TIMEOUT = -4
SG_E_CUDA = -5
ABI_VERSION = 2
EXPORTS = ("eemd_sg_version", "eemd_sg_conv", "eemd_sg_pack", "eemd_sg_wgrad", "eemd_sg_loss", "eemd_sg_adam",
           "eemd_sg_bias", "eemd_sg_scale", "eemd_sg_prepare", "eemd_sg_combine", "eemd_sg_stat_count")

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
    lib.eemd_sg_pack.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32,
                                 c_void_p]
    lib.eemd_sg_bias.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p]
    lib.eemd_sg_scale.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_void_p]
    lib.eemd_sg_prepare.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_int32, c_int32, c_int32, c_int32, c_void_p]
    lib.eemd_sg_combine.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32, c_double,
                                    c_double, c_int32, c_void_p, c_void_p, c_void_p]
    lib.eemd_sg_stat_count.restype = c_int32
    lib.eemd_sg_wgrad.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32,
                                  c_int32, c_int32, c_int32, c_int32, c_void_p, c_int64, c_void_p]
    lib.eemd_sg_loss.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32,
                                 c_int32, c_int32, c_int32, c_float, c_void_p, c_void_p]
    lib.eemd_sg_adam.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_float, c_float, c_float,
                                 c_float, c_int32, c_float, c_void_p, c_void_p]
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


def pack(w, wpk, n_rows, c, nv, cv, transpose=False, project=False):
    _check(load().eemd_sg_pack(_p(w), _p(wpk), n_rows, c, nv, cv, int(transpose), int(project), _stream()),
           "eemd_sg_pack")


def bias(b, out, n_rows, nv, project=False):
    _check(load().eemd_sg_bias(_p(b), _p(out), n_rows, nv, int(project), _stream()), "eemd_sg_bias")


def scale(x, out, S, N):
    _check(load().eemd_sg_scale(_p(x), _p(out), S, N, _stream()), "eemd_sg_scale")


def prepare(imf_sum, mode_count, x, scl, out, S, N, K, C, imf_sum2=None, mode_count2=None):
    _check(load().eemd_sg_prepare(_p(imf_sum), _p(mode_count), _p(imf_sum2), _p(mode_count2), _p(x), _p(scl),
                                  _p(out), S, N, K, C, _stream()), "eemd_sg_prepare")


def stat_count() -> int:
    return int(load().eemd_sg_stat_count())


def combine(imf_sum, mode_count, x, scl, net_out, imfs_out, resid_out, partial, chunks, S, N, K, C, P,
            recon_bound, io_bound, metrics, fallback, io_relative=True):
    _check(load().eemd_sg_combine(_p(imf_sum), _p(mode_count), _p(x), _p(scl), _p(net_out), _p(imfs_out),
                                  _p(resid_out), _p(partial), chunks, S, N, K, C, P, float(recon_bound),
                                  float(io_bound), int(io_relative), _p(metrics), _p(fallback), _stream()),
           "eemd_sg_combine")


def wgrad(dy, x, dw, db, B, T, n_rows, c, nv, cv, dil, tensor_cores=True, err=None, spin_limit=0):
    _check(load().eemd_sg_wgrad(_p(dy), _p(x), _p(dw), _p(db), B, T, n_rows, c, nv, cv, dil, int(tensor_cores),
                                _p(err), spin_limit, _stream()), "eemd_sg_wgrad")


def loss(out, base, target, dout, acc, B, T, c, cv, margin, project=False, delta=0.0, weights=None):
    _check(load().eemd_sg_loss(_p(out), _p(base), _p(target), _p(dout), _p(acc), B, T, c, cv, margin,
                               int(project), float(delta), _p(weights), _stream()), "eemd_sg_loss")


def adam(p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8, max_norm=0.0, work=None):
    _check(load().eemd_sg_adam(_p(p), _p(g), _p(m), _p(v), p.numel(), lr, b1, b2, eps, step, float(max_norm),
                               _p(work), _stream()), "eemd_sg_adam")
