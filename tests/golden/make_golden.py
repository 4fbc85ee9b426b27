"""Generate the golden fixtures from the reference implementation itself.

Run in a container that holds the reference checkout (misureaudio/EEMD4CUDA):

    python tests/golden/make_golden.py <reference checkout>

It imports the reference's emd_ref.py / refsignal.py / emd_gpu.py (the last
under numba's CUDA simulator, NUMBA_ENABLE_CUDASIM=1, so the reference GPU
kernel runs on the CPU for small N) and writes:

  known_answers.json  integer results (mode counts, sift counts, per-sift knot
                      counts) and per-IMF checksums of the reference's
                      decompositions on the workloads used by the tests
  small_cases.npz     full float64 outputs of small cases (N <= 8192)

Nothing under tests/ reads the reference at test time; only these files.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def checksum(a: np.ndarray) -> dict:
    a = np.asarray(a, dtype=np.float64)
    idx = np.linspace(0, len(a) - 1, 16).astype(int)
    return {"sum": float(a.sum()), "sumsq": float((a * a).sum()),
            "maxabs": float(np.abs(a).max()), "idx": idx.tolist(),
            "vals": [float(v) for v in a[idx]]}


SIM_SCRIPT = r"""
import os, sys, json
os.environ['NUMBA_ENABLE_CUDASIM'] = '1'
sys.path.insert(0, sys.argv[1])
import numpy as np
import emd_gpu as G
d = np.load(sys.argv[2])
X = d['X']; E, N = X.shape; MAXIMF = int(d['maximf']); tau = float(d['tau']); ms = int(d['max_sifts'])
K = max(16, N // 2)
kern = G.get_full_kernel(N, K, MAXIMF, 32)
resid = np.empty((E, N)); h = np.empty((E, N)); out = np.zeros((E, MAXIMF, N))
eu = np.empty((E, N)); W = np.empty((E, 10 * K))
ns = np.zeros(E, np.int32); nm = np.zeros(E, np.int32)
kern[E, 32](X.copy(), resid, h, out, eu, W, ns, nm, tau, ms, 4)
np.savez(sys.argv[3], out=out, nsift=ns, nmode=nm)
"""


def run_numba_sim(ref: str, X: np.ndarray, maximf: int, tau: float, max_sifts: int):
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        src = Path(td) / "in.npz"
        dst = Path(td) / "out.npz"
        script = Path(td) / "sim.py"
        np.savez(src, X=X, maximf=maximf, tau=tau, max_sifts=max_sifts)
        script.write_text(SIM_SCRIPT)
        subprocess.run([sys.executable, str(script), ref, str(src), str(dst)], check=True)
        d = np.load(dst)
        return d["out"].copy(), d["nsift"].copy(), d["nmode"].copy()


def main(ref: str):
    sys.path.insert(0, ref)
    sys.path.insert(0, str(REPO))
    import emd_ref as R
    from refsignal import make_ref_signal
    from eemd4cuda_b200 import signals
    from eemd4cuda_b200.emd_par import make_reference_sweep

    ka: dict = {}
    small: dict = {}

    # --- reference sweep: our restated generator reproduces refsignal bit-exactly
    xr, _ = make_ref_signal()
    xs, _ = make_reference_sweep()
    ka["sweep_identical_to_refsignal"] = bool(np.array_equal(xr, xs))

    def emd_record(x, **kw):
        # emd_ref.emd_1d with the knot counts of every sift (same loop, counted)
        imfs, resid, st = R.emd_1d(x, **kw)
        return imfs, resid, st

    # --- config A: sweep[:110250], E=1, tau .25, 50 sifts, max_imf 16
    xA = xr[:110250]
    imfs, resid, st = emd_record(xA, tau=0.25, max_sifts=50, max_imf=16)
    ka["A"] = {"n_modes": st["n_modes"], "total_sifts": st["total_sifts"],
               "per_mode_sifts": st["per_mode_sifts"],
               "imf": [checksum(m) for m in imfs], "resid": checksum(resid)}

    # --- config B: 8 trials, default_rng(7) perturbation 0.2 std (test_phase3_gates.py:80-82)
    rng = np.random.default_rng(7)
    XB = xA[None, :] + 0.2 * np.std(xA) * rng.standard_normal((8, len(xA)))
    B = {"n_modes": [], "total_sifts": [], "per_mode_sifts": [], "imf0": [], "imf_last": []}
    for e in range(8):
        im, rs, s2 = R.emd_1d(XB[e], tau=0.25, max_sifts=50, max_imf=16)
        B["n_modes"].append(s2["n_modes"])
        B["total_sifts"].append(s2["total_sifts"])
        B["per_mode_sifts"].append(s2["per_mode_sifts"])
        B["imf0"].append(checksum(im[0]))
        B["imf_last"].append(checksum(im[-1]))
    ka["B"] = B

    # --- plain EMD workload: N=8192 @ 8 kHz, mirror ends, 10 IMFs, SD<0.2 or 10 sifts
    x1 = signals.plain_emd_8k()
    im1, rs1, st1 = R.emd_1d(x1, tau=0.2, max_sifts=10, max_imf=10, end="mirror")
    ka["plain8k_mirror"] = {"n_modes": st1["n_modes"], "total_sifts": st1["total_sifts"],
                            "per_mode_sifts": st1["per_mode_sifts"],
                            "recon": float(np.max(np.abs(x1 - (np.sum(im1, axis=0) + rs1))))}
    small["plain8k_x"] = x1
    small["plain8k_imfs"] = np.array(im1)
    small["plain8k_resid"] = rs1

    # --- A1: one sift on the 2048-sample chirp (test_emd_gpu.py:89-102)
    N1 = 2048
    t1 = np.arange(N1)
    r1 = np.random.default_rng(1)
    f1 = 0.01 + 0.05 * t1 / N1
    xa1 = (np.sin(2 * np.pi * np.cumsum(f1)) + 0.3 * np.sin(2 * np.pi * 0.013 * t1)
           + 0.1 * r1.standard_normal(N1))
    eu, _ = R.envelope(t1.astype(float), xa1, "max", "natural")
    el, _ = R.envelope(t1.astype(float), xa1, "min", "natural")
    small["a1_x"] = xa1
    small["a1_h1"] = xa1 - 0.5 * (eu + el)
    for end in ("natural", "mirror"):
        im, rs, s3 = R.emd_1d(xa1, tau=0.25, max_sifts=50, end=end)
        small[f"chirp2048_{end}_imfs"] = np.array(im)
        small[f"chirp2048_{end}_resid"] = rs
        ka[f"chirp2048_{end}"] = {"n_modes": s3["n_modes"], "total_sifts": s3["total_sifts"],
                                  "per_mode_sifts": s3["per_mode_sifts"]}

    # --- pathological spacing chirp (test_phase3_gates.py:200-206)
    x8 = signals.modulated_chirp()
    kmax = np.where((x8[1:-1] > x8[:-2]) & (x8[1:-1] > x8[2:]))[0] + 1
    kmin = np.where((x8[1:-1] < x8[:-2]) & (x8[1:-1] < x8[2:]))[0] + 1
    k = np.sort(np.concatenate([kmax, kmin]))
    hsp = np.diff(k.astype(float))
    im8, rs8, s8 = R.emd_1d(x8, tau=0.25, max_sifts=50, max_imf=16)
    ka["G8"] = {"cv": float(hsp.std() / hsp.mean()), "n_modes": s8["n_modes"],
                "total_sifts": s8["total_sifts"], "per_mode_sifts": s8["per_mode_sifts"],
                "imf": [checksum(m) for m in im8]}

    # --- stage fixture: two tones 100/105 Hz, E=1 CPU (audio_eemd/tests/test_eemd_stage.py:8-16)
    xt, sr = signals.two_tones()
    imt, rst, stt = R.emd_1d(xt, tau=0.25, max_sifts=50)
    ka["two_tones"] = {"n_modes": stt["n_modes"], "total_sifts": stt["total_sifts"],
                       "per_mode_sifts": stt["per_mode_sifts"]}

    # --- the reference numba GPU kernel (emd_gpu.py) under the CUDA simulator
    N = 512
    rs_ = np.random.default_rng(3)
    tt = np.arange(N)
    xs_ = np.sin(2 * np.pi * 0.03 * tt) + 0.5 * np.sin(2 * np.pi * 0.11 * tt) + 0.1 * rs_.standard_normal(N)
    XS = xs_[None, :] + 0.2 * np.std(xs_) * rs_.standard_normal((3, N))
    out, ns, nm = run_numba_sim(ref, XS, 6, 0.25, 50)
    small["numba_X"] = XS
    small["numba_out"] = out
    ka["numba_sim"] = {"nsift": ns.tolist(), "nmode": nm.tolist(), "maximf": 6, "tau": 0.25,
                       "max_sifts": 50}

    # --- DSBT mirror of the reference (audit_eemd/test_block_thomas.py dsbt_solve) on two systems
    sys.path.insert(0, str(Path(ref) / "audit_eemd"))
    import importlib.util
    spec = importlib.util.spec_from_file_location("tbt_audit", str(Path(ref) / "audit_eemd" / "test_block_thomas.py"))
    tbt = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tbt)
    for kind in ("uniform", "cv15"):
        tm, ym = tbt.synth_knots(kind)
        d, l, u, H, n = tbt.build_system(tm)
        r = tbt.rhs_of(tm, ym, H, n)
        small[f"dsbt_{kind}_tm"] = tm
        small[f"dsbt_{kind}_ym"] = ym
        small[f"dsbt_{kind}_x"] = tbt.dsbt_solve(d, l, u, r)
        small[f"dsbt_{kind}_exact"] = R.thomas(d, l, u, r)

    (HERE / "known_answers.json").write_text(json.dumps(ka, indent=1))
    np.savez_compressed(HERE / "small_cases.npz", **small)
    print("wrote", HERE / "known_answers.json", HERE / "small_cases.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
