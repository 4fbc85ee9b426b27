"""Generate the spectra fixtures from the reference implementation itself.

    python tests/golden/make_spectra_golden.py <reference checkout>

Loads the reference's audio_eemd/spectra.py (its stft_block and hilbert_if,
on scipy.signal) as a module and runs them on small seeded IMF-like signals;
writes tests/golden/spectra_cases.npz.  Nothing under tests/ reads the
reference at test time.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def signals(N, seed, sr):
    """three IMF-like rows: an AM tone, a chirp, band-limited noise"""
    t = np.arange(N) / sr
    rng = np.random.default_rng(seed)
    a = (1 + 0.3 * np.sin(2 * np.pi * 3 * t)) * np.sin(2 * np.pi * 440 * t + 0.2)
    b = 0.5 * np.sin(2 * np.pi * (200 * t + 800 * t * t))
    w = rng.standard_normal(N)
    k = np.exp(-0.5 * (np.arange(-40, 41) / 10.0) ** 2)
    c = np.convolve(w, k / k.sum(), mode="same") * np.sin(2 * np.pi * 1500 * t)
    return np.vstack([a, b, c])


CASES = [  # (name, N, seed, sr, nperseg, noverlap)
    ("a", 3000, 0, 8000, 256, None),
    ("b", 4097, 1, 16000, 512, 384),
    ("c", 2048, 2, 48000, 2048, None),
]


def main(ref_dir: str):
    spec = importlib.util.spec_from_file_location("ref_spectra", Path(ref_dir) / "audio_eemd" / "spectra.py")
    sp = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sp)
    out = {}
    for name, N, seed, sr, nper, nov in CASES:
        X = signals(N, seed, sr)
        out[f"{name}_x"] = X
        out[f"{name}_params"] = np.array([N, sr, nper, -1 if nov is None else nov], dtype=np.int64)
        for r in range(X.shape[0]):
            f, t, Z = sp.stft_block(X[r], sr, nperseg=nper, noverlap=nov)
            w, A = sp.hilbert_if(X[r], sr)
            out[f"{name}_{r}_Z"] = Z
            out[f"{name}_{r}_if"] = w
            out[f"{name}_{r}_amp"] = A
            st = sp.if_stats(w)
            out[f"{name}_{r}_ifstats"] = np.array([np.nan if st["median"] is None else st["median"],
                                                   np.nan if st["iqr"] is None else st["iqr"], st["n_pos_frac"]])
        out[f"{name}_f"] = f
        out[f"{name}_t"] = t
        print(name, Z.shape)
    np.savez_compressed(HERE / "spectra_cases.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
