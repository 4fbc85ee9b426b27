"""Audio decode, segmentation and a pipelined segment-by-segment EEMD.

The reference decodes with soundfile (audio_eemd/audio_io.py:71-176), which
is not installed in this image; this module reads FLAC streams through its
own decoder (libeemd_flac.so, include/eemd_flac.h: RFC 9639, every frame's
CRCs checked and the stream's MD5 signature compared) and RIFF/WAVE files
itself (PCM 8/16/24/32-bit and IEEE float 32/64-bit, any channel count) into
the same float64 [frames, channels] array soundfile returns (PCM scaled by
2^-(bits-1), unsigned 8-bit centred first) and keeps the reference's
segment rules: `AudioFile.to_mono` (mean over channels), `select_segment`
(seconds or samples, stop exclusive, typed SegmentError codes) and
`resolve_segment` (whole file up to 30 s, else the first 10 s).

`decompose_segments` runs the EEMD of consecutive segments of a long signal
with the host and the device overlapped: while the engine decomposes segment
k, segment k+1 is copied to the device on a copy stream and the modes of
segment k-1 are copied back and written (results.AsyncWriter).
"""
from __future__ import annotations

import ctypes
import hashlib
import struct
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

DEFAULT_MAX_FILE_SEC = 30.0
DEFAULT_SEGMENT_SEC = 10.0


class AudioError(Exception):
    """Unreadable or unsupported audio file."""

    def __init__(self, message: str, code: str = "audio.unreadable"):
        super().__init__(message)
        self.code = code


class SegmentError(Exception):
    """Bad segment limits or unit."""

    def __init__(self, message: str, code: str = "segment.bad_limits"):
        super().__init__(message)
        self.code = code


@dataclass
class AudioFile:
    path: Path
    sr: int
    channels: int
    frames: int
    duration: float
    fmt: str
    subtype: str
    x: np.ndarray  # float64 [frames, channels]
    meta: dict = field(default_factory=dict)

    def to_mono(self) -> np.ndarray:
        """Mean over channels."""
        if self.channels == 1:
            return self.x[:, 0]
        return self.x.mean(axis=1)


def _decode(fmt_tag, bits, data, channels):
    if fmt_tag == 1:  # PCM
        if bits == 8:
            v = (np.frombuffer(data, dtype=np.uint8).astype(np.float64) - 128.0) / 128.0
            sub = "PCM_U8"
        elif bits == 16:
            v = np.frombuffer(data, dtype="<i2").astype(np.float64) / 32768.0
            sub = "PCM_16"
        elif bits == 24:
            b = np.frombuffer(data, dtype=np.uint8).reshape(-1, 3).astype(np.int32)
            iv = b[:, 0] | (b[:, 1] << 8) | (b[:, 2] << 16)
            iv = np.where(iv >= 1 << 23, iv - (1 << 24), iv)
            v = iv.astype(np.float64) / float(1 << 23)
            sub = "PCM_24"
        elif bits == 32:
            v = np.frombuffer(data, dtype="<i4").astype(np.float64) / float(1 << 31)
            sub = "PCM_32"
        else:
            raise AudioError(f"unsupported PCM bit depth {bits}", "audio.unsupported")
    elif fmt_tag == 3:  # IEEE float
        if bits == 32:
            v = np.frombuffer(data, dtype="<f4").astype(np.float64)
            sub = "FLOAT"
        elif bits == 64:
            v = np.frombuffer(data, dtype="<f8").astype(np.float64)
            sub = "DOUBLE"
        else:
            raise AudioError(f"unsupported float bit depth {bits}", "audio.unsupported")
    else:
        raise AudioError(f"unsupported WAVE format tag {fmt_tag}", "audio.unsupported")
    frames = len(v) // channels
    return v[:frames * channels].reshape(frames, channels), sub


_FLAC = None


class FlacInfo(ctypes.Structure):
    """Mirror of `eemd_flac_stream_info` (include/eemd_flac.h)."""

    _fields_ = [("sample_rate", ctypes.c_int32), ("channels", ctypes.c_int32),
                ("bits_per_sample", ctypes.c_int32), ("min_block", ctypes.c_int32),
                ("max_block", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("total_frames", ctypes.c_int64), ("first_frame_offset", ctypes.c_int64),
                ("md5", ctypes.c_uint8 * 16)]


def _flac_lib():
    global _FLAC
    if _FLAC is None:
        path = Path(__file__).resolve().parent / "lib" / "libeemd_flac.so"
        if not path.exists():
            raise AudioError(f"FLAC decoder library not found at {path}; build it with "
                             "`python -m eemd4cuda_b200.build`", "audio.unsupported")
        lib = ctypes.CDLL(str(path))
        lib.eemd_flac_info.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(FlacInfo)]
        lib.eemd_flac_info.restype = ctypes.c_int32
        lib.eemd_flac_decode.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int64)]
        lib.eemd_flac_decode.restype = ctypes.c_int32
        lib.eemd_flac_strerror.argtypes = [ctypes.c_int32]
        lib.eemd_flac_strerror.restype = ctypes.c_char_p
        _FLAC = lib
    return _FLAC


def decode_flac(raw: bytes):
    """(int32 samples [frames, channels], FlacInfo) of a FLAC stream; AudioError
    on a malformed stream, a CRC mismatch or an MD5 signature mismatch."""
    lib = _flac_lib()
    info = FlacInfo()
    rc = lib.eemd_flac_info(raw, len(raw), ctypes.byref(info))
    if rc:
        raise AudioError(f"not a readable FLAC stream: {lib.eemd_flac_strerror(rc).decode()}")
    total = int(info.total_frames)
    if total == 0:
        # length not recorded: every frame takes at least 8 bytes (header,
        # one subframe header, CRC-16) and holds at most max_block samples
        total = (len(raw) // 8 + 1) * int(info.max_block)
    out = np.empty((total, int(info.channels)), dtype=np.int32)
    got = ctypes.c_int64(0)
    rc = lib.eemd_flac_decode(raw, len(raw), out.ctypes.data, total, ctypes.byref(got))
    if rc:
        raise AudioError(f"FLAC decode failed after {got.value} frames: {lib.eemd_flac_strerror(rc).decode()}")
    x = out[:got.value]
    md5 = bytes(info.md5)
    if any(md5):
        nb = (int(info.bits_per_sample) + 7) // 8
        le = x.astype("<i4").view(np.uint8).reshape(-1, 4)[:, :nb]
        if hashlib.md5(le.tobytes()).digest() != md5:
            raise AudioError("FLAC stream's MD5 signature does not match its decoded samples")
    return x, info


def _load_flac(p: Path, raw: bytes) -> AudioFile:
    x, info = decode_flac(raw)
    bps = int(info.bits_per_sample)
    if x.shape[0] == 0:
        raise AudioError(f"unexpected sample array shape {x.shape} from {p}")
    v = x.astype(np.float64) / float(1 << (bps - 1))
    sr, ch, frames = int(info.sample_rate), int(info.channels), int(x.shape[0])
    sub = {8: "PCM_S8", 16: "PCM_16", 24: "PCM_24"}.get(bps, f"PCM_{bps}")
    meta = {"format": "FLAC", "subtype": sub, "samplerate": sr, "channels": ch, "frames": frames,
            "duration_s": frames / float(sr)}
    return AudioFile(path=p, sr=sr, channels=ch, frames=frames, duration=frames / float(sr), fmt="FLAC",
                     subtype=sub, x=v, meta=meta)


def load_audio(path) -> AudioFile:
    """Read a FLAC or RIFF/WAVE file fully into memory (AudioError on failure)."""
    p = Path(path)
    try:
        raw = p.read_bytes()
    except OSError as e:
        raise AudioError(f"cannot read audio file {p}: {e}") from e
    if raw[:4] == b"fLaC":
        return _load_flac(p, raw)
    if len(raw) < 12 or raw[:4] != b"RIFF" or raw[8:12] != b"WAVE":
        raise AudioError(f"cannot read audio file {p}: not a FLAC or RIFF/WAVE file")
    pos, fmt, data = 12, None, None
    while pos + 8 <= len(raw):
        cid, size = raw[pos:pos + 4], struct.unpack("<I", raw[pos + 4:pos + 8])[0]
        body = raw[pos + 8:pos + 8 + size]
        if cid == b"fmt ":
            fmt = body
        elif cid == b"data":
            data = body
        pos += 8 + size + (size & 1)
    if fmt is None or data is None or len(fmt) < 16:
        raise AudioError(f"cannot read audio file {p}: missing fmt or data chunk")
    tag, channels, sr, _, _, bits = struct.unpack("<HHIIHH", fmt[:16])
    if tag == 0xFFFE and len(fmt) >= 26:  # WAVE_FORMAT_EXTENSIBLE: the sub-format's first two bytes
        tag = struct.unpack("<H", fmt[24:26])[0]
    if channels < 1 or sr < 1:
        raise AudioError(f"cannot read audio file {p}: bad header")
    x, sub = _decode(tag, bits, data, channels)
    if x.shape[0] == 0:
        raise AudioError(f"unexpected sample array shape {x.shape} from {p}")
    frames = x.shape[0]
    meta = {"format": "WAV", "subtype": sub, "samplerate": int(sr), "channels": int(channels),
            "frames": int(frames), "duration_s": frames / float(sr)}
    return AudioFile(path=p, sr=int(sr), channels=int(channels), frames=int(frames), duration=frames / float(sr),
                     fmt="WAV", subtype=sub, x=x, meta=meta)


def select_segment(a: AudioFile, limits: Sequence[float], unit: str = "s") -> np.ndarray:
    """Mono float64 segment [limits[0], limits[1]) (stop exclusive), in seconds or samples."""
    mono = a.to_mono()
    n = len(mono)
    if unit == "s":
        s0 = int(round(limits[0] * a.sr))
        s1 = int(round(limits[1] * a.sr))
    elif unit == "samples":
        s0, s1 = int(limits[0]), int(limits[1])
    else:
        raise SegmentError(f"unit must be 's' or 'samples', got {unit!r}", "segment.bad_unit")
    if s0 < 0 or s1 <= s0 or s1 > n:
        raise SegmentError(f"limits [{limits[0]}, {limits[1]}] (unit={unit!r}) out of range for {n} samples "
                           "(stop exclusive)", "segment.out_of_range")
    return mono[s0:s1].copy()


def resolve_segment(a: AudioFile, limits=None, unit="s", max_file_sec=DEFAULT_MAX_FILE_SEC):
    """(xseg, limits, unit, defaulted): the whole file up to max_file_sec, else its first 10 s."""
    defaulted = False
    if limits is None:
        if a.duration <= max_file_sec:
            limits, unit = [0.0, a.duration], "s"
        else:
            limits, unit = [0.0, DEFAULT_SEGMENT_SEC], "s"
            defaulted = True
    return select_segment(a, limits, unit), limits, unit, defaulted


def segment_bounds(n: int, n_seg: int) -> list:
    """[start, stop) of consecutive segments of n_seg samples covering n
    samples; a last segment under 8 samples (too short for EMD) joins its
    predecessor."""
    if n < 1:
        raise ValueError("empty signal")
    bounds = [(s, min(s + n_seg, n)) for s in range(0, n, n_seg)]
    if bounds[-1][1] - bounds[-1][0] < 8 and len(bounds) > 1:
        bounds[-2] = (bounds[-2][0], bounds[-1][1])
        bounds.pop()
    return bounds


def decompose_segments(x, sr, segment_s=DEFAULT_SEGMENT_SEC, *, E=64, eps=0.2, tau=0.25, max_sifts=50,
                       max_imf=8, seed=0, dtype=np.float32, outdir=None, return_modes=True):
    """EEMD of x cut into consecutive segments of segment_s seconds (the last
    may be shorter; one under 8 samples joins its predecessor), host and
    device overlapped.  Returns a list of (imfs [n_modes, n] float64,
    residual [n]) per segment (empty with return_modes=False); with
    `outdir`, segment k's imfs.npz is written to outdir/seg_<k>/ by a
    background writer.  Segment k uses noise seed `seed + k`."""
    import torch

    from . import _lib as L
    from . import emd_par as M
    from . import results

    x = np.asarray(x, dtype=np.float64)
    bounds = segment_bounds(len(x), max(1, int(round(segment_s * sr))))
    dev = torch.device("cuda", torch.cuda.current_device())
    dt = np.dtype(dtype)
    tdt = torch.float32 if dt == np.float32 else torch.float64
    comp = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    longest = max(b - a for a, b in bounds)
    slots = M.imf_slots(longest, max_imf)
    pin = [torch.empty((longest,), dtype=tdt).pin_memory() for _ in range(2)]
    xd = [torch.empty((longest,), dtype=tdt, device=dev) for _ in range(2)]
    ready = [torch.cuda.Event() for _ in range(2)]
    writer = results.AsyncWriter() if outdir is not None else None
    out = []

    def stage(k):
        a, b = bounds[k]
        buf = k & 1
        pin[buf][:b - a].copy_(torch.from_numpy(x[a:b].astype(dt)))
        with torch.cuda.stream(copy):
            xd[buf][:b - a].copy_(pin[buf][:b - a], non_blocking=True)
            ready[buf].record(copy)

    stage(0)
    for k, (a, b) in enumerate(bounds):
        n = b - a
        buf = k & 1
        comp.wait_event(ready[buf])
        p = M.make_params(dtype=dt, noise_mode=L.EEMD_NOISE_PHILOX, eps=eps, seed=seed + k, tau=tau,
                          max_sifts=max_sifts, max_imf=slots)
        ws = torch.empty((L.workspace_size(p, [n], E, False),), dtype=torch.uint8, device=dev)
        imf_sum = torch.zeros((slots * n,), dtype=torch.float64, device=dev)
        cnt = torch.zeros((slots,), dtype=torch.int32, device=dev)
        mean = torch.empty((slots, n), dtype=torch.float64, device=dev)
        resid = torch.empty((n,), dtype=torch.float64, device=dev)
        nm = torch.empty((1,), dtype=torch.int32, device=dev)
        xk = xd[buf][:n]
        L.run(p, xk, [n], 0, E, ws, imf_sum=imf_sum, mode_count=cnt)
        L.finalize(p, xk, [n], imf_sum, cnt, mean, resid, nm)
        if k + 1 < len(bounds):
            # the next segment's upload overlaps this segment's kernels; its
            # buffers were last used by segment k-1, finished at the sync below
            stage(k + 1)
        m = int(nm.item())
        if writer is not None:
            d = Path(outdir) / f"seg_{k:04d}"
            d.mkdir(parents=True, exist_ok=True)
            t = (np.arange(n) + a) / float(sr)
            writer.submit(d, x[a:b], t, mean[:m], resid, m, dict(E=E, segment=k))
        if return_modes:
            out.append((mean[:m].cpu().numpy(), resid.cpu().numpy()))
    if writer is not None:
        writer.close()
    return out
