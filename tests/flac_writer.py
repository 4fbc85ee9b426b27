"""A small FLAC encoder for the decoder's tests (test infrastructure).

No FLAC file or encoder exists in this environment (soundfile / libsndfile is
not installed and the reference's FLAC fixtures are not part of its
checkout), so the tests write their own streams, following the format of
RFC 9639: STREAMINFO with the MD5 of the samples, frame headers with CRC-8,
subframes of every kind the decoder handles (CONSTANT, VERBATIM, FIXED 0-4,
LPC with quantised coefficients, wasted bits), partitioned Rice residuals
with 4- and 5-bit parameters and the escape to raw binary, every stereo
decorrelation mode, fixed and variable blocking, coded block sizes and
sample rates, and the frame CRC-16.  Each choice is explicit so that a test
can force every path; the decoder must return the encoder's input exactly.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field

import numpy as np


class BitWriter:
    def __init__(self):
        self.bits: list[int] = []

    def u(self, v: int, k: int):
        v = int(v)
        assert 0 <= v < (1 << k) or k == 0, (v, k)
        self.bits.extend((v >> (k - 1 - i)) & 1 for i in range(k))

    def s(self, v: int, k: int):
        v = int(v)
        assert -(1 << (k - 1)) <= v < (1 << (k - 1)), (v, k)
        self.u(v & ((1 << k) - 1), k)

    def unary(self, q: int):
        self.bits.extend([0] * int(q))
        self.bits.append(1)

    def align(self):
        while len(self.bits) % 8:
            self.bits.append(0)

    def tobytes(self) -> bytes:
        assert len(self.bits) % 8 == 0
        out = bytearray()
        for i in range(0, len(self.bits), 8):
            b = 0
            for bit in self.bits[i:i + 8]:
                b = (b << 1) | bit
            out.append(b)
        return bytes(out)


def crc8(data: bytes) -> int:
    c = 0
    for x in data:
        c ^= x
        for _ in range(8):
            c = ((c << 1) ^ 0x07) & 0xFF if c & 0x80 else (c << 1) & 0xFF
    return c


def crc16(data: bytes) -> int:
    c = 0
    for x in data:
        c ^= x << 8
        for _ in range(8):
            c = ((c << 1) ^ 0x8005) & 0xFFFF if c & 0x8000 else (c << 1) & 0xFFFF
    return c


def coded_number(v: int) -> bytes:
    """The UTF-8-style coding of frame and sample numbers (up to 36 bits)."""
    if v < 0x80:
        return bytes([v])
    for n in range(2, 8):
        payload = 6 * (n - 1) + (7 - n if n < 7 else 0)
        if v < (1 << payload):
            break
    else:
        raise ValueError(v)
    tail = [0x80 | ((v >> (6 * i)) & 0x3F) for i in range(n - 1)][::-1]
    lead_bits = v >> (6 * (n - 1))
    lead = ((0xFF << (8 - n)) & 0xFF) | lead_bits if n < 7 else 0xFE
    return bytes([lead] + tail)


@dataclass
class Sub:
    """How one subframe is coded."""
    kind: str = "fixed"          # constant | verbatim | fixed | lpc
    order: int = 2               # fixed: 0..4; lpc: 1..32
    precision: int = 12          # lpc coefficient bits
    shift: int = 9               # lpc quantisation shift
    porder: int = 2              # Rice partition order
    rice5: bool = False          # 5-bit Rice parameters (coding method 1)
    escape_parts: tuple = ()     # partitions written as raw binary
    wasted: bool = True          # use wasted bits when the samples allow


def _rice_param(u: np.ndarray, maxp: int) -> int:
    if len(u) == 0:
        return 0
    m = float(np.mean(u))
    k = 0
    while k < maxp - 1 and (1 << (k + 1)) <= m:
        k += 1
    return k


def _residual(w: BitWriter, res: np.ndarray, bs: int, order: int, sub: Sub):
    w.u(1 if sub.rice5 else 0, 2)
    w.u(sub.porder, 4)
    parts = 1 << sub.porder
    assert bs % parts == 0 and bs // parts >= order
    esc = 31 if sub.rice5 else 15
    pbits = 5 if sub.rice5 else 4
    i = 0
    for part in range(parts):
        cnt = bs // parts - (order if part == 0 else 0)
        r = res[i:i + cnt].astype(np.int64)
        i += cnt
        if part in sub.escape_parts:
            nb = 0
            if cnt:
                mx = int(max(np.max(r), -np.min(r) - 1, 0))
                nb = mx.bit_length() + 1
            w.u(esc, pbits)
            w.u(nb, 5)
            for v in r:
                w.s(int(v), nb) if nb else None
            continue
        u = np.where(r >= 0, 2 * r, -2 * r - 1)
        k = _rice_param(u, esc)
        w.u(k, pbits)
        for x in u:
            x = int(x)
            w.unary(x >> k)
            w.u(x & ((1 << k) - 1), k)


def _lpc_coefs(x: np.ndarray, order: int, precision: int, shift: int) -> np.ndarray:
    """Levinson-Durbin on the block's autocorrelation, quantised."""
    xf = x.astype(np.float64)
    r = np.array([np.dot(xf[:len(xf) - k], xf[k:]) for k in range(order + 1)])
    r[0] = r[0] * (1 + 1e-9) + 1e-9
    a = np.zeros(order)
    e = r[0]
    for i in range(order):
        acc = r[i + 1] - np.dot(a[:i], r[i:0:-1])
        k = acc / e
        a_new = a.copy()
        a_new[i] = k
        a_new[:i] = a[:i] - k * a[:i][::-1]
        a = a_new
        e *= (1 - k * k)
    lim = (1 << (precision - 1)) - 1
    return np.clip(np.round(a * (1 << shift)), -lim - 1, lim).astype(np.int64)


def subframe(w: BitWriter, s: np.ndarray, bps: int, sub: Sub):
    s = s.astype(np.int64)
    bs = len(s)
    wasted = 0
    if sub.wasted and sub.kind != "constant" and np.any(s):
        while wasted < bps - 1 and not np.any(s & ((1 << (wasted + 1)) - 1)):
            wasted += 1
    w.u(0, 1)
    code = {"constant": 0, "verbatim": 1}.get(sub.kind)
    if sub.kind == "fixed":
        code = 8 + sub.order
    elif sub.kind == "lpc":
        code = 32 + sub.order - 1
    w.u(code, 6)
    if wasted:
        w.u(1, 1)
        w.unary(wasted - 1)
    else:
        w.u(0, 1)
    v = s >> wasted
    eb = bps - wasted
    if sub.kind == "constant":
        assert np.all(s == s[0])
        w.s(int(s[0]), bps)
    elif sub.kind == "verbatim":
        for x in v:
            w.s(int(x), eb)
    elif sub.kind == "fixed":
        o = sub.order
        for x in v[:o]:
            w.s(int(x), eb)
        res = v.copy()
        for _ in range(o):
            res = np.diff(res)
        _residual(w, np.asarray(res), bs, o, sub)
    else:
        o = sub.order
        coef = _lpc_coefs(v, o, sub.precision, sub.shift)
        for x in v[:o]:
            w.s(int(x), eb)
        w.u(sub.precision - 1, 4)
        w.s(sub.shift, 5)
        for c in coef:
            w.s(int(c), sub.precision)
        pred = np.zeros(bs, dtype=np.int64)
        for j in range(o):
            pred[o:] += coef[j] * v[o - 1 - j:bs - 1 - j]
        res = v[o:] - (pred[o:] >> sub.shift)
        _residual(w, np.concatenate([np.zeros(o, dtype=np.int64), res])[o:], bs, o, sub)


_RATE_CODES = {88200: 1, 176400: 2, 192000: 3, 8000: 4, 16000: 5, 22050: 6, 24000: 7, 32000: 8,
               44100: 9, 48000: 10, 96000: 11}
_SIZE_CODES = {8: 1, 12: 2, 16: 4, 20: 5, 24: 6, 32: 7}


@dataclass
class Frame:
    mode: str = "independent"    # independent | left_side | side_right | mid_side
    subs: list = field(default_factory=list)   # one Sub per channel (repeated if shorter)
    bs_code: str = "auto"        # auto | explicit8 | explicit16
    rate_code: str = "table"     # table | streaminfo | khz8 | hz16 | tenhz16
    size_code: str = "table"     # table | streaminfo


def encode(x: np.ndarray, sr: int, bps: int, blocks: list, frames: list | None = None,
           variable: bool = False) -> bytes:
    """x: int [n, channels]; blocks: block sizes summing to n; frames: one
    Frame per block (default: independent channels, FIXED order 2)."""
    x = np.asarray(x, dtype=np.int64)
    n, C = x.shape
    assert sum(blocks) == n
    frames = frames or [Frame() for _ in blocks]
    out = bytearray(b"fLaC")
    si = BitWriter()
    si.u(min(blocks[:-1] or blocks) if len(blocks) > 1 else blocks[0], 16)
    si.u(max(blocks), 16)
    si.u(0, 24)
    si.u(0, 24)
    si.u(sr, 20)
    si.u(C - 1, 3)
    si.u(bps - 1, 5)
    si.u(n, 36)
    nb = (bps + 7) // 8
    raw = b"".join(int(v).to_bytes(nb, "little", signed=True) for v in x.reshape(-1))
    for b in hashlib.md5(raw).digest():
        si.u(b, 8)
    out += bytes([0x80 | 0, 0, 0, 34]) + si.tobytes()
    pos = 0
    for fi, (bs, fr) in enumerate(zip(blocks, frames)):
        blk = x[pos:pos + bs]
        hw = BitWriter()
        hw.u(0x3FFE, 14)
        hw.u(0, 1)
        hw.u(1 if variable else 0, 1)
        table = {192: 1, 576: 2, 1152: 3, 2304: 4, 4608: 5, 256: 8, 512: 9, 1024: 10, 2048: 11,
                 4096: 12, 8192: 13, 16384: 14, 32768: 15}
        if fr.bs_code == "auto" and bs in table:
            bsc = table[bs]
        elif fr.bs_code == "explicit8" or (fr.bs_code == "auto" and bs <= 256):
            bsc = 6
        else:
            bsc = 7
        hw.u(bsc, 4)
        if fr.rate_code == "table":
            src = _RATE_CODES[sr]
        else:
            src = {"streaminfo": 0, "khz8": 12, "hz16": 13, "tenhz16": 14}[fr.rate_code]
        hw.u(src, 4)
        chc = {"independent": C - 1, "left_side": 8, "side_right": 9, "mid_side": 10}[fr.mode]
        hw.u(chc, 4)
        hw.u(_SIZE_CODES[bps] if fr.size_code == "table" else 0, 3)
        hw.u(0, 1)
        head = bytearray(hw.tobytes())
        head += coded_number(pos if variable else fi)
        if bsc == 6:
            head.append(bs - 1)
        elif bsc == 7:
            head += (bs - 1).to_bytes(2, "big")
        if src == 12:
            head.append(sr // 1000)
        elif src == 13:
            head += sr.to_bytes(2, "big")
        elif src == 14:
            head += (sr // 10).to_bytes(2, "big")
        head.append(crc8(bytes(head)))
        if fr.mode == "independent":
            chans, widths = [blk[:, c] for c in range(C)], [bps] * C
        else:
            L, R = blk[:, 0], blk[:, 1]
            if fr.mode == "left_side":
                chans, widths = [L, L - R], [bps, bps + 1]
            elif fr.mode == "side_right":
                chans, widths = [L - R, R], [bps + 1, bps]
            else:
                chans, widths = [(L + R) >> 1, L - R], [bps, bps + 1]
        sw = BitWriter()
        subs = fr.subs or [Sub()]
        for c, (sig, wd) in enumerate(zip(chans, widths)):
            subframe(sw, sig, wd, subs[c % len(subs)])
        sw.align()
        body = bytes(head) + sw.tobytes()
        out += body + crc16(body).to_bytes(2, "big")
        pos += bs
    return bytes(out)
