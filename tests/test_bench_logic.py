"""Host-side arithmetic of bench.py (CPU): the algorithmic-byte count of a
k_emd launch and the per-workload measured traffic."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402


def test_algorithmic_bytes_by_hand():
    # 2 tasks (1 signal of 1000 samples, 2 trials), float32 (b = 4)
    klog = np.full((2, 3, 4, 2), -1, dtype=np.int32)
    klog[0, 0, :2] = [[100, 99], [90, 91]]   # task 0, IMF 0: two sifts
    klog[0, 1, :1] = [[40, 41]]              # task 0, IMF 1: one sift
    klog[1, 0, :1] = [[120, 118]]            # task 1, IMF 0: one sift
    nmode = np.array([2, 1], dtype=np.int32)
    n, b = 1000, 4
    per_knot = 3 * (4 + b) + 16
    want = (2 * n * b                                   # task 0 input / perturbed input
            + 3 * (3 * n * b) + (199 + 181 + 81) * per_knot + 2 * (4 * n * b)
            + 2 * n * b                                 # task 1
            + 3 * n * b + 238 * per_knot + 4 * n * b)
    got = bench.emd_algorithmic_bytes(klog, nmode, [n], 2, b)
    assert got == want


def test_measured_traffic_per_workload():
    full, src = bench.measured_traffic("harmonic48k", 100)
    assert isinstance(full, int) and full > 0
    assert set(src) == {"capture", "engine_sha256", "traffic_matches_build"}
    assert bench.measured_traffic("harmonic48k", 7)[0] == full  # a launch capture is not rescaled
    a64, a32 = bench.measured_traffic("amfm4m", 64)[0], bench.measured_traffic("amfm4m", 32)[0]
    assert a64 > 0 and abs(a64 - 2 * a32) <= 1
    assert bench.measured_traffic("plain8k", 1) == (None, None)
    # the flag follows the engine source the capture ran
    assert len(bench.engine_source_sha256()) == 64


def test_spectra_launch_count():
    """The spectra line's launch count follows the FFT plan of libeemd_spectra.so:
    4096 = 4^6 in one shared-memory launch, 48000 = 200 x 240 and 8192 =
    64 x 128 as four-step pairs, 2^25 as 13 global passes, 4099 (prime)
    through Bluestein's 16384-point transforms (4 + 3 * 2), 37 through
    Bluestein's 128-point ones (4 + 3 * 1); the Hilbert call of 48000 is 5
    launches, an STFT of 4096-sample frames one."""
    assert bench.fft4_split(48000) == (200, 240)
    assert bench.fft4_split(65536) == (256, 256)
    assert bench.fft4_split(4096) is None
    assert bench.fft_passes(48000) == 2
    assert bench.fft_passes(4096) == 1
    assert bench.fft_passes(8192) == 2
    assert bench.fft_passes(1 << 25) == 13
    assert bench.fft_passes(4099) == 4 + 3 * 2
    assert bench.fft_passes(37) == 4 + 3 * 1
    assert bench.spectra_launches(48000, 4096) == 2 * 1 + 5
    assert bench.spectra_launches(48000, 8192) == 2 * (2 + 2) + 5


def test_companion_summary_and_failures(monkeypatch):
    """The headline line's brief companion lines: the summary keeps the value,
    end-to-end figure and roofline of a workload's line, and a companion that
    fails (here: no GPU in this process's child) becomes an error entry
    instead of an exception."""
    line = {"metric": "m", "value": 1.5, "unit": "u", "ms_per_step": 2.0, "steps": 1, "dtype": "f64",
            "config": {"workload": "w"}, "e2e": {"value": 1.2}, "clocks": {"sm_mhz": 1965.0},
            "roofline": {"kernel": "k_emd", "achieved": 10.0, "peak": 100.0, "unit": "GB/s", "frac": 0.1,
                         "traffic": 5}}
    s = bench.companion_summary(line)
    assert s["value"] == 1.5 and s["e2e"] == 1.2 and s["workload"] == "w" and s["clocks_sm_mhz"] == 1965.0
    assert s["roofline"] == {"kernel": "k_emd", "achieved": 10.0, "peak": 100.0, "unit": "GB/s", "frac": 0.1}
    monkeypatch.setattr(bench, "COMPANIONS", (("plain8k", 120),))
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "")
    res = bench.run_companions()
    assert set(res) == {"plain8k"} and "error" in res["plain8k"]


def test_reference_arm_line():
    """`bench.py --impl reference` (the reference's CPU path on the host
    cores, no GPU) prints one JSON line with the GPU arm's metric and unit,
    a cpu_baseline describing the run and an e2e entry with no host-device
    bytes."""
    import json
    import subprocess

    r = subprocess.run([sys.executable, str(Path(bench.__file__)), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 3 and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "harmonic_clicks_48k_eemd"


def test_reference_arm_under_two_ranks():
    """Launched like the multi-GPU bench (torchrun, two ranks, 127.0.0.1):
    rank 0 alone runs the reference's CPU path and prints the one line; the
    other rank exits 0 without work."""
    import json
    import socket
    import subprocess

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(bench.__file__)),
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
