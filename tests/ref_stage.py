"""The reference's own stage adapter, unchanged, plugged onto this engine.

`audio_eemd/eemd_stage.py` (the caller of the hot path in the reference)
prepends its `_EMD4CUDA_DIR` to sys.path and runs `import emd_par`
(eemd_stage.py:27-33).  `load()` imports that very file from the reference
installed in baseline/_ref (python baseline/install_reference.py <checkout>;
the installed file is byte-identical to the checkout's) and sets the module
attribute `_EMD4CUDA_DIR` to eemd4cuda_b200/compat, the way a user of the
reference points it at this engine without editing the file.  Tests that use
it are skipped when the reference is not installed.

`import audio_eemd` itself needs soundfile (audio_io.py:13), which this
environment lacks, so the stage module is loaded from its file; it has no
relative imports.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "baseline" / "_ref"
STAGE = REF / "audio_eemd" / "eemd_stage.py"
COMPAT = ROOT / "eemd4cuda_b200" / "compat"


def load(monkeypatch):
    if not STAGE.exists():
        pytest.skip("the reference is not installed in baseline/_ref "
                    "(python baseline/install_reference.py <reference checkout>)")
    name = "_reference_eemd_stage"
    spec = importlib.util.spec_from_file_location(name, STAGE)
    mod = importlib.util.module_from_spec(spec)
    # dataclasses resolve the module through sys.modules while the class body runs
    monkeypatch.setitem(sys.modules, name, mod)
    spec.loader.exec_module(mod)
    monkeypatch.setattr(mod, "_EMD4CUDA_DIR", COMPAT)
    # the stage's own `import emd_par` must find the compat module, not a cached one
    monkeypatch.delitem(sys.modules, "emd_par", raising=False)
    monkeypatch.setattr(sys, "path", list(sys.path))
    return mod
