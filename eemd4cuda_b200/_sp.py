"""ctypes binding of libeemd_spectra.so (the C ABI of include/eemd_spectra.h)."""
from __future__ import annotations

import ctypes
from ctypes import c_double, c_int32, c_int64, c_size_t, c_void_p
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
SP_OK = 0
ABI_VERSION = 1
EXPORTS = ("eemd_sp_version", "eemd_sp_fft_workspace", "eemd_sp_fft", "eemd_sp_hilbert_workspace",
           "eemd_sp_hilbert_if", "eemd_sp_stft_shape", "eemd_sp_stft_workspace", "eemd_sp_stft")
_ERR = {-1: "bad argument", -2: "workspace too small", -5: "CUDA error"}

_lib = None


class SpectraError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: {_ERR.get(status, 'status')} ({status})")
        self.status = status


def lib_path() -> Path:
    return LIB_DIR / "libeemd_spectra.so"


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        raise RuntimeError(f"{path} is missing: build it with `python -m eemd4cuda_b200.build`")
    lib = ctypes.CDLL(str(path))
    lib.eemd_sp_version.restype = c_int32
    if lib.eemd_sp_version() != ABI_VERSION:
        raise RuntimeError("libeemd_spectra.so ABI version mismatch")
    lib.eemd_sp_fft_workspace.argtypes = [c_int32, c_int64, ctypes.POINTER(c_size_t)]
    lib.eemd_sp_fft.argtypes = [c_void_p, c_void_p, c_int32, c_int64, c_int32, c_void_p, c_size_t, c_void_p]
    lib.eemd_sp_hilbert_workspace.argtypes = [c_int32, c_int64, ctypes.POINTER(c_size_t)]
    lib.eemd_sp_hilbert_if.argtypes = [c_void_p, c_int32, c_int64, c_double, c_void_p, c_void_p, c_void_p, c_size_t,
                                       c_void_p]
    lib.eemd_sp_stft_shape.argtypes = [c_int64, c_int32, c_int32, ctypes.POINTER(c_int32), ctypes.POINTER(c_int32)]
    lib.eemd_sp_stft_workspace.argtypes = [c_int32, c_int64, c_int32, c_int32, ctypes.POINTER(c_size_t)]
    lib.eemd_sp_stft.argtypes = [c_void_p, c_int32, c_int64, c_int32, c_int32, c_void_p, c_void_p, c_size_t,
                                 c_void_p]
    for f in EXPORTS[1:]:
        getattr(lib, f).restype = c_int32
    _lib = lib
    return lib


def _check(rc, where):
    if rc != SP_OK:
        raise SpectraError(rc, where)


def _stream():
    import torch
    return c_void_p(torch.cuda.current_stream().cuda_stream)


def hilbert_workspace(M, N) -> int:
    b = c_size_t()
    _check(load().eemd_sp_hilbert_workspace(M, N, ctypes.byref(b)), "eemd_sp_hilbert_workspace")
    return b.value


def hilbert_if(x, M, N, sr, freq, amp, ws):
    _check(load().eemd_sp_hilbert_if(c_void_p(x.data_ptr()), M, N, float(sr), c_void_p(freq.data_ptr()),
                                     c_void_p(amp.data_ptr()), c_void_p(ws.data_ptr()), ws.numel(), _stream()),
           "eemd_sp_hilbert_if")


def stft_shape(N, nperseg, noverlap):
    F, T = c_int32(), c_int32()
    _check(load().eemd_sp_stft_shape(N, nperseg, noverlap, ctypes.byref(F), ctypes.byref(T)), "eemd_sp_stft_shape")
    return F.value, T.value


def stft_workspace(M, N, nperseg, noverlap) -> int:
    b = c_size_t()
    _check(load().eemd_sp_stft_workspace(M, N, nperseg, noverlap, ctypes.byref(b)), "eemd_sp_stft_workspace")
    return b.value


def stft(x, M, N, nperseg, noverlap, Z, ws):
    _check(load().eemd_sp_stft(c_void_p(x.data_ptr()), M, N, nperseg, noverlap, c_void_p(Z.data_ptr()),
                               c_void_p(ws.data_ptr()), ws.numel(), _stream()), "eemd_sp_stft")


def fft_device(z, sign=-1):
    """FFT of every row of a complex128 CUDA tensor [M, N] (sign -1: numpy.fft.fft;
    +1: the unnormalised inverse), through eemd_sp_fft; returns a new tensor."""
    import torch
    lib = load()
    z = z.contiguous()
    M, N = int(z.shape[0]), int(z.shape[1])
    nb = c_size_t(0)
    _check(lib.eemd_sp_fft_workspace(M, N, ctypes.byref(nb)), "eemd_sp_fft_workspace")
    ws = torch.empty((max(int(nb.value), 1),), dtype=torch.uint8, device=z.device)
    out = torch.empty_like(z)
    _check(lib.eemd_sp_fft(z.data_ptr(), out.data_ptr(), M, N, int(sign), ws.data_ptr(), int(nb.value), _stream()),
           "eemd_sp_fft")
    return out
