import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def known():
    return json.loads((GOLDEN / "known_answers.json").read_text())


@pytest.fixture(scope="session")
def small():
    d = np.load(GOLDEN / "small_cases.npz")
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def sweep():
    from eemd4cuda_b200.emd_par import make_reference_sweep
    x, _ = make_reference_sweep()
    return x


def checksum_close(a, ck, rtol=1e-12):
    """Compare an array with a checksum record of tests/golden/make_golden.py."""
    a = np.asarray(a, dtype=np.float64)
    scale = max(ck["maxabs"], 1e-300)
    vals = a[np.asarray(ck["idx"])]
    err = max(np.max(np.abs(vals - np.asarray(ck["vals"]))) / scale,
              abs(float((a * a).sum()) - ck["sumsq"]) / max(ck["sumsq"], 1e-300),
              abs(float(a.sum()) - ck["sum"]) / (scale * len(a)))
    return err <= rtol, err
