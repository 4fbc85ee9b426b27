"""WAV decode and the reference's segment rules (audio_eemd/audio_io.py:52-176)."""
import struct

import numpy as np
import pytest

from eemd4cuda_b200 import audio


def write_wav(path, data, sr, tag, bits):
    """data: [frames, channels] already in the file's sample type"""
    frames, ch = data.shape
    body = np.ascontiguousarray(data).tobytes()
    if bits == 24:
        iv = data.astype(np.int32).reshape(-1)
        b = np.stack([iv & 255, (iv >> 8) & 255, (iv >> 16) & 255], axis=1).astype(np.uint8)
        body = b.tobytes()
    block = ch * bits // 8
    fmt = struct.pack("<HHIIHH", tag, ch, sr, sr * block, block, bits)
    riff = b"WAVE" + b"fmt " + struct.pack("<I", len(fmt)) + fmt + b"data" + struct.pack("<I", len(body)) + body
    path.write_bytes(b"RIFF" + struct.pack("<I", len(riff)) + riff)


@pytest.mark.parametrize("bits,tag,dtype,scale", [(16, 1, "<i2", 32768.0), (24, 1, None, float(1 << 23)),
                                                  (32, 1, "<i4", float(1 << 31)), (32, 3, "<f4", 1.0),
                                                  (64, 3, "<f8", 1.0)])
def test_decode_scales_like_libsndfile(tmp_path, bits, tag, dtype, scale):
    rng = np.random.default_rng(bits + tag)
    if tag == 1:
        lim = int(scale)
        ints = rng.integers(-lim, lim, size=(500, 2))
        data = ints.astype(dtype) if dtype else ints
        want = ints.astype(np.float64) / scale
    else:
        data = rng.uniform(-1, 1, size=(500, 2)).astype(dtype)
        want = data.astype(np.float64)
    p = tmp_path / "a.wav"
    write_wav(p, data, 44100, tag, bits)
    a = audio.load_audio(p)
    assert a.sr == 44100 and a.channels == 2 and a.frames == 500
    assert np.array_equal(a.x, want)
    assert np.array_equal(a.to_mono(), want.mean(axis=1))


def test_unsigned_8_bit(tmp_path):
    data = np.array([[0], [128], [255]], dtype=np.uint8)
    p = tmp_path / "u8.wav"
    write_wav(p, data, 8000, 1, 8)
    a = audio.load_audio(p)
    assert np.array_equal(a.x[:, 0], (np.array([0, 128, 255]) - 128) / 128.0)


def test_segments_and_errors(tmp_path):
    data = (np.arange(8000 * 40) % 100).astype("<i2").reshape(-1, 1)
    p = tmp_path / "long.wav"
    write_wav(p, data, 8000, 1, 16)
    a = audio.load_audio(p)
    seg, limits, unit, defaulted = audio.resolve_segment(a)
    assert defaulted and len(seg) == 80000 and limits == [0.0, 10.0]
    assert len(audio.select_segment(a, [100, 300], "samples")) == 200
    with pytest.raises(audio.SegmentError) as e:
        audio.select_segment(a, [5, 1], "s")
    assert e.value.code == "segment.out_of_range"
    with pytest.raises(audio.SegmentError) as e:
        audio.select_segment(a, [0, 1], "ms")
    assert e.value.code == "segment.bad_unit"
    (tmp_path / "bad.wav").write_bytes(b"not audio")
    with pytest.raises(audio.AudioError):
        audio.load_audio(tmp_path / "bad.wav")


def test_segment_bounds():
    assert audio.segment_bounds(20500, 8000) == [(0, 8000), (8000, 16000), (16000, 20500)]
    assert audio.segment_bounds(16005, 8000) == [(0, 8000), (8000, 16005)]  # a 5-sample sliver joins
    assert audio.segment_bounds(100, 8000) == [(0, 100)]
    with pytest.raises(ValueError):
        audio.segment_bounds(0, 8000)
