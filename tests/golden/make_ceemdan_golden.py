"""Generate the CEEMDAN fixtures from the reference implementation itself.

    python tests/golden/make_ceemdan_golden.py <reference checkout>

Imports the reference's emd_ref.py and runs its ceemdan() serially
(parallel=False) on small seeded signals, and its emd_1d() on the stage-0
noise rows for their mode counts; writes tests/golden/ceemdan_cases.npz.
Nothing under tests/ reads the reference at test time.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def signal(N, seed):
    t = np.arange(N) / 8000.0
    rng = np.random.default_rng(seed)
    return (0.8 * np.sin(2 * np.pi * 50 * t) + 0.5 * np.sin(2 * np.pi * 400 * t + 0.3)
            + 0.3 * np.sin(2 * np.pi * (1000 * t + 500 * t * t / t[-1])) + 0.05 * rng.standard_normal(N))


CASES = [  # (name, N, signal seed, E, eps, ceemdan seed, tau, max_sifts, end)
    ("a", 1024, 0, 8, 0.2, 3, 0.25, 50, "natural"),
    ("b", 2048, 1, 12, 0.2, 5, 0.2, 10, "natural"),
    ("c", 1536, 2, 6, 0.3, 7, 0.25, 50, "mirror"),
]


def main(ref_dir: str):
    sys.path.insert(0, ref_dir)
    import emd_ref  # the reference module

    out = {}
    for name, N, sseed, E, eps, seed, tau, ms, end in CASES:
        x = signal(N, sseed)
        c, r, st = emd_ref.ceemdan(x, E=E, eps=eps, parallel=False, seed=seed, tau=tau, max_sifts=ms, end=end)
        W = emd_ref._gen_noise(E, N, seed)
        nm = [emd_ref.emd_1d(W[e] + np.zeros(N), tau=tau, max_sifts=ms, min_extrema=4, end=end)[2]["n_modes"]
              for e in range(E)]
        out[f"{name}_x"] = x
        out[f"{name}_c"] = c
        out[f"{name}_r"] = r
        out[f"{name}_noise_modes"] = np.array(nm, dtype=np.int32)
        out[f"{name}_params"] = np.array([N, E, eps, seed, tau, ms, 0 if end == "natural" else 1], dtype=np.float64)
        print(name, "n_imfs", st["n_imfs"], "noise modes", sorted(set(nm)))
    np.savez_compressed(HERE / "ceemdan_cases.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
