"""FLAC decode (libeemd_flac.so through eemd4cuda_b200.audio) against streams
written by tests/flac_writer.py: every subframe kind, Rice coding method,
escape partition, wasted-bits case, stereo decorrelation mode, coded block
size and sample rate, fixed and variable blocking must come back exactly, the
stream's MD5 signature must match, and damaged streams must be refused
(audio_eemd/audio_io.py:71-103 reads the same files through soundfile)."""
import numpy as np
import pytest

from eemd4cuda_b200 import audio
from flac_writer import Frame, Sub, encode


def _signal(n, C, bps, seed):
    rng = np.random.default_rng(seed)
    t = np.arange(n)
    amp = (1 << (bps - 1)) - 1
    x = np.empty((n, C), dtype=np.int64)
    for c in range(C):
        s = 0.5 * np.sin(2 * np.pi * (0.003 + 0.002 * c) * t) + 0.3 * np.sin(2 * np.pi * 0.041 * t + c)
        s += 0.05 * rng.standard_normal(n)
        x[:, c] = np.clip(np.round(s * amp), -amp - 1, amp)
    return x


def _roundtrip(tmp_path, x, sr, bps, blocks, frames=None, variable=False):
    data = encode(x, sr, bps, blocks, frames, variable)
    got, info = audio.decode_flac(data)
    assert info.sample_rate == sr and info.channels == x.shape[1] and info.bits_per_sample == bps
    assert np.array_equal(got, x)
    p = tmp_path / "t.flac"
    p.write_bytes(data)
    a = audio.load_audio(p)
    assert a.fmt == "FLAC" and a.sr == sr and a.frames == len(x) and a.channels == x.shape[1]
    assert np.array_equal(a.x, x / float(1 << (bps - 1)))
    return data


@pytest.mark.parametrize("bps", [8, 16, 24])
def test_fixed_orders_and_rice(tmp_path, bps):
    x = _signal(4096 * 3 + 1000, 1, bps, 1)
    frames = [Frame(subs=[Sub("fixed", order=o, porder=p)]) for o, p in ((0, 0), (1, 3), (4, 6))]
    frames.append(Frame(subs=[Sub("fixed", order=3, porder=3, rice5=True)]))
    _roundtrip(tmp_path, x, 44100, bps, [4096, 4096, 4096, 1000], frames)


def test_constant_verbatim_lpc_and_escape(tmp_path):
    x = _signal(2048 * 5, 1, 16, 2)
    x[0:2048] = 1234  # a constant block
    frames = [Frame(subs=[Sub("constant")]),
              Frame(subs=[Sub("verbatim")]),
              Frame(subs=[Sub("lpc", order=8, precision=12, shift=10, porder=4)]),
              Frame(subs=[Sub("lpc", order=32, precision=15, shift=13, porder=5, escape_parts=(0, 7))]),
              Frame(subs=[Sub("fixed", order=2, porder=2, escape_parts=(1,), rice5=True)])]
    _roundtrip(tmp_path, x, 48000, 16, [2048] * 5, frames)


def test_wasted_bits(tmp_path):
    x = _signal(4096 * 2, 2, 16, 3) & ~0xF  # four zero low bits in every sample
    frames = [Frame(subs=[Sub("fixed", order=2)]), Frame(subs=[Sub("lpc", order=4, precision=14, shift=12)])]
    _roundtrip(tmp_path, x, 44100, 16, [4096, 4096], frames)


@pytest.mark.parametrize("mode", ["independent", "left_side", "side_right", "mid_side"])
def test_stereo_modes(tmp_path, mode):
    x = _signal(4608 * 2 + 300, 2, 24, 4)
    frames = [Frame(mode=mode, subs=[Sub("fixed", order=2, porder=1), Sub("lpc", order=12, precision=13, shift=11)])
              for _ in range(3)]
    _roundtrip(tmp_path, x, 96000, 24, [4608, 4608, 300], frames)


def test_coded_block_sizes_rates_and_variable_blocking(tmp_path):
    x = _signal(192 + 200 + 3000 + 576 + 50000, 3, 16, 5)
    blocks = [192, 200, 3000, 576, 50000]
    frames = [Frame(rate_code="streaminfo", size_code="streaminfo"),
              Frame(bs_code="explicit8", rate_code="khz8"),
              Frame(bs_code="explicit16", rate_code="hz16"),
              Frame(rate_code="tenhz16"),
              Frame(bs_code="explicit16")]
    # the sample-number coding reaches 3 bytes with variable blocking
    _roundtrip(tmp_path, x, 32000, 16, blocks, frames, variable=True)


def test_damaged_streams_are_refused(tmp_path):
    x = _signal(4096 * 2, 1, 16, 6)
    data = encode(x, 44100, 16, [4096, 4096])
    bad = bytearray(data)
    bad[len(data) // 2] ^= 0x10  # a bit inside the first or second frame
    with pytest.raises(audio.AudioError):
        audio.decode_flac(bytes(bad))
    with pytest.raises(audio.AudioError):
        audio.decode_flac(data[: len(data) - 5])  # truncated last frame
    with pytest.raises(audio.AudioError):
        audio.decode_flac(b"fLaX" + data[4:])
    p = tmp_path / "x.flac"
    p.write_bytes(bytes(bad))
    with pytest.raises(audio.AudioError) as ei:
        audio.load_audio(p)
    assert ei.value.code == "audio.unreadable"


def test_segment_of_a_flac_file(tmp_path):
    """The reference's segment rules on a decoded FLAC file (mono mean, stop exclusive)."""
    x = _signal(48000, 2, 16, 7)
    p = tmp_path / "s.flac"
    p.write_bytes(encode(x, 48000, 16, [4096] * 11 + [48000 - 4096 * 11]))
    a = audio.load_audio(p)
    seg = audio.select_segment(a, [0.25, 0.5])
    assert np.array_equal(seg, (x[12000:24000] / 32768.0).mean(axis=1))
