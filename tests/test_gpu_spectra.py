"""The spectra stage on the GPU (libeemd_spectra.so) against fixtures made by
the reference's own audio_eemd/spectra.py and against the CPU oracle."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import spectra_oracle as SP

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from eemd4cuda_b200 import spectra  # noqa: E402


@pytest.fixture(scope="module")
def golden():
    d = np.load(GOLDEN / "spectra_cases.npz")
    return {k: d[k] for k in d.files}


def steady(amp, frac=1e-3):
    """samples whose analytic-signal magnitude (and its neighbours') is not
    near zero: elsewhere the phase, hence the frequency, is ill-conditioned"""
    ok = amp > frac * amp.max()
    return ok & np.roll(ok, 1) & np.roll(ok, -1)


@pytest.mark.parametrize("name", ["a", "b", "c"])
def test_spectra_match_reference(golden, name):
    N, sr, nper, nov = golden[f"{name}_params"].tolist()
    nov = None if nov < 0 else nov
    X = golden[f"{name}_x"]
    # the batched call: all rows at once
    f, t, Z = spectra.stft_block(X, sr, nperseg=nper, noverlap=nov)
    w, A = spectra.hilbert_if(X, sr)
    assert np.allclose(f, golden[f"{name}_f"], rtol=0, atol=1e-9)
    assert np.allclose(t, golden[f"{name}_t"], rtol=0, atol=1e-12)
    for r in range(X.shape[0]):
        Zr = golden[f"{name}_{r}_Z"]
        assert Z[r].shape == Zr.shape
        assert np.max(np.abs(Z[r] - Zr)) <= 1e-11 * np.max(np.abs(Zr))
        Ar, wr = golden[f"{name}_{r}_amp"], golden[f"{name}_{r}_if"]
        assert np.max(np.abs(A[r] - Ar)) <= 1e-11 * np.max(Ar)
        m = steady(Ar)
        assert np.max(np.abs(w[r] - wr)[m]) <= 1e-6 * sr
        st = spectra.if_stats(w[r])
        ref = golden[f"{name}_{r}_ifstats"]
        assert abs(st["n_pos_frac"] - ref[2]) <= 2.0 / N
        assert abs(st["median"] - ref[0]) <= 1e-6 * sr
    # one row at a time gives the same as the batch
    f1, t1, Z1 = spectra.stft_block(X[1], sr, nperseg=nper, noverlap=nov)
    w1, A1 = spectra.hilbert_if(X[1], sr)
    assert np.max(np.abs(Z1 - Z[1])) <= 1e-13 * np.max(np.abs(Z1))
    assert np.max(np.abs(A1 - A[1])) <= 1e-13 * np.max(A1)


def test_spectra_of_imfs_48k_against_the_oracle():
    """Ten IMF-sized rows of 48 000 samples, device-resident in and out."""
    rng = np.random.default_rng(5)
    sr, N = 48000, 48000
    t = np.arange(N) / sr
    rows = [np.sin(2 * np.pi * (f0 * t + 30 * t * t)) * (1 + 0.2 * np.sin(2 * np.pi * 2 * t))
            for f0 in rng.uniform(30, 9000, 10)]
    X = np.vstack(rows)
    Xd = torch.from_numpy(X).cuda()
    w, A = spectra.hilbert_if_device(Xd, sr)
    f, tt, Z = spectra.stft_device(Xd, sr, nperseg=4096)
    assert w.is_cuda and Z.is_cuda
    w, A, Z = w.cpu().numpy(), A.cpu().numpy(), Z.cpu().numpy()
    for r in range(10):
        ow, oA = SP.hilbert_if(X[r], sr)
        assert np.max(np.abs(A[r] - oA)) <= 1e-10 * np.max(oA)
        m = steady(oA)
        # the oracle differentiates a cumulative phase of up to ~1e5 rad; allow its rounding
        assert np.max(np.abs(w[r] - ow)[m]) <= 1e-6 * sr
        _, _, oZ = SP.stft(X[r], sr, 4096)
        assert np.max(np.abs(Z[r] - oZ)) <= 1e-11 * np.max(np.abs(oZ))


@pytest.mark.parametrize("N", [1, 2, 3, 5, 8, 30, 37, 100, 1001, 2048, 4097, 6144, 7168, 48000, 65536])
def test_own_fft_against_numpy(N):
    """eemd_sp_fft (Stockham radix 4/2/3/5/odd primes <= 31, Bluestein for
    larger primes: 37, 4097 = 17 x 241) against numpy.fft on 3 rows, both signs;
    lengths up to 4096 run as one shared-memory launch per row (37's Bluestein
    transforms of 128 too), longer ones as the four-step transform of two
    shared-memory launches (6144 = 64 x 96, 7168 = 64 x 112, 48000 =
    200 x 240, 65536 = 256 x 256, 4097's Bluestein transforms of 8192)."""
    from eemd4cuda_b200 import _sp
    rng = np.random.default_rng(N)
    x = rng.standard_normal((3, N)) + 1j * rng.standard_normal((3, N))
    z = torch.from_numpy(x).cuda()
    f = _sp.fft_device(z, -1).cpu().numpy()
    ref = np.fft.fft(x, axis=1)
    assert np.max(np.abs(f - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
    b = _sp.fft_device(z, +1).cpu().numpy()
    refb = np.fft.ifft(x, axis=1) * N
    assert np.max(np.abs(b - refb)) <= 1e-13 * max(1.0, np.max(np.abs(refb)))


def test_fft_beyond_the_four_step_limit():
    """A row of 2^25 (longer than 4096 x 4096) runs as global Stockham passes."""
    from eemd4cuda_b200 import _sp
    N = 1 << 25
    rng = np.random.default_rng(25)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    f = _sp.fft_device(torch.from_numpy(x[None, :]).cuda(), -1).cpu().numpy()[0]
    ref = np.fft.fft(x)
    assert np.max(np.abs(f - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("nper", [256, 1000, 4096, 8192])
def test_stft_frame_lengths_against_oracle(nper):
    """The STFT's one-launch shared-memory form (frames of up to 4096 samples
    with radix 4/2/3/5 factors) and its global-pass form (8192) against the
    oracle's restatement of the reference's scipy call."""
    rng = np.random.default_rng(nper)
    sr, N = 48000, 20000
    X = rng.standard_normal((2, N))
    f, t, Z = spectra.stft_block(X, sr, nperseg=nper)
    for r in range(2):
        of, ot, oZ = SP.stft(X[r], sr, nper)
        assert np.allclose(f, of) and np.allclose(t, ot)
        assert np.max(np.abs(Z[r] - oZ)) <= 1e-11 * np.max(np.abs(oZ))


def tones(rng, rows, N):
    """rows of three tones of random frequency and phase, slight noise"""
    t = np.arange(N, dtype=float)
    out = np.zeros((rows, N))
    for r in range(rows):
        for _ in range(3):
            out[r] += rng.uniform(0.2, 1.0) * np.cos(2 * np.pi * rng.uniform(0.002, 0.2) * t + rng.uniform(0, 6.3))
        out[r] += 0.01 * rng.standard_normal(N)
    return out


@pytest.mark.parametrize("N", [2, 3, 5, 8, 31, 33, 1001, 4097])
def test_hilbert_short_and_odd_lengths_against_oracle(N):
    """The analytic signal's one-sided weights for even and odd N (a single
    Nyquist bin only when N is even) down to two samples: amplitude and
    instantaneous frequency against the oracle's restatement of
    scipy.signal.hilbert + unwrap + gradient (audio_eemd/spectra.py:18-30)."""
    rng = np.random.default_rng(N)
    sr = 48000
    X = tones(rng, 3, N)
    w, A = spectra.hilbert_if(X, sr)
    assert w.shape == A.shape == (3, N)
    for r in range(3):
        ow, oA = SP.hilbert_if(X[r], sr)
        assert np.max(np.abs(A[r] - oA)) <= 1e-12 * max(1.0, np.max(oA)), r
        m = steady(oA)
        if m.any():
            assert np.max(np.abs(w[r] - ow)[m]) <= 1e-6 * sr, r


@pytest.mark.parametrize("N,nper,nov", [(5000, 1000, 333), (4096, 512, 384), (777, 64, 1), (20000, 4096, 0)])
def test_stft_other_overlaps_against_oracle(N, nper, nov):
    """Hops other than half a frame (a third, an eighth, one sample short of
    a whole frame, no overlap): frame count, axes and bins against the
    oracle."""
    rng = np.random.default_rng(N + nov)
    sr = 48000
    X = tones(rng, 2, N)
    f, t, Z = spectra.stft_block(X, sr, nperseg=nper, noverlap=nov)
    for r in range(2):
        of, ot, oZ = SP.stft(X[r], sr, nper, nov)
        assert Z[r].shape == oZ.shape
        assert np.allclose(f, of) and np.allclose(t, ot)
        assert np.max(np.abs(Z[r] - oZ)) <= 1e-11 * np.max(np.abs(oZ))


def test_stft_of_a_signal_shorter_than_the_frame():
    """nperseg above the signal length (audio_eemd/spectra.py:25-29 over
    scipy.signal.stft): the default overlap, half the requested frame, is
    then not below the cut frame, a ValueError; with an explicit overlap a
    warning and frames of the signal's length."""
    rng = np.random.default_rng(3)
    sr, N = 48000, 1000
    X = tones(rng, 2, N)
    with pytest.warns(UserWarning, match="nperseg"), pytest.raises(ValueError, match="noverlap"):
        spectra.stft_block(X, sr, nperseg=4096)
    with pytest.warns(UserWarning, match="nperseg"):
        f, t, Z = spectra.stft_block(X, sr, nperseg=4096, noverlap=300)
    for r in range(2):
        of, ot, oZ = SP.stft(X[r], sr, N, 300)
        assert Z[r].shape == oZ.shape
        assert np.allclose(f, of) and np.allclose(t, ot)
        assert np.max(np.abs(Z[r] - oZ)) <= 1e-11 * np.max(np.abs(oZ))


def test_large_rows_through_pageable_copies():
    """Rows whose results exceed the pinned-transfer size (two rows of 2^23
    samples: 128 MB per result array) move through pageable copies, with the
    same results as the oracle."""
    assert 2 * (1 << 23) * 8 > spectra.PINNED_BYTES
    rng = np.random.default_rng(23)
    sr, N = 48000, 1 << 23
    X = tones(rng, 2, N)
    w, A = spectra.hilbert_if(X, sr)
    for r in range(2):
        ow, oA = SP.hilbert_if(X[r], sr)
        assert np.max(np.abs(A[r] - oA)) <= 1e-10 * np.max(oA)
        m = steady(oA)
        assert np.max(np.abs(w[r] - ow)[m]) <= 1e-6 * sr
