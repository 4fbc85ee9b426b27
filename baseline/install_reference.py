"""Install the unmodified reference (misureaudio/EEMD4CUDA) into baseline/_ref.

    python baseline/install_reference.py <reference checkout>

The reference ships no packaging metadata (no setup.py / pyproject.toml), so
pip cannot install the checkout as it is.  This script copies the checkout to
a temporary directory, adds a minimal pyproject.toml there that names the
reference's own modules (the CPU ground truth emd_ref.py, the public API
emd_par.py, the numba kernel module emd_gpu.py, refsignal.py and the
audio_eemd package), and runs the offline pip install

    pip install --no-index --no-build-isolation --find-links /opt/wheelhouse \
        --target baseline/_ref <temporary copy>

No reference file is changed: the installed modules are byte-identical to the
checkout's (checked at the end).  baseline/_ref is git-ignored; it travels
with the working tree to the machines that run bench.py --impl reference and
the drop-in tests of the reference's own stage adapter.
"""
from __future__ import annotations

import filecmp
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

MODULES = ["emd_ref", "emd_par", "emd_gpu", "refsignal"]
PACKAGE = "audio_eemd"

PYPROJECT = """\
[build-system]
requires = ["setuptools"]
build-backend = "setuptools.build_meta"

[project]
name = "eemd4cuda-reference"
version = "0.0.0"

[tool.setuptools]
py-modules = {modules}
packages = ["{package}"]
"""


def main(ref: Path) -> int:
    out = Path(__file__).resolve().parent / "_ref"
    if out.exists():
        shutil.rmtree(out)
    with tempfile.TemporaryDirectory() as tmp:
        src = Path(tmp) / "src"
        src.mkdir()
        for m in MODULES:
            shutil.copy2(ref / f"{m}.py", src / f"{m}.py")
        shutil.copytree(ref / PACKAGE, src / PACKAGE, ignore=shutil.ignore_patterns("__pycache__"))
        (src / "pyproject.toml").write_text(
            PYPROJECT.format(modules="[" + ", ".join(f'"{m}"' for m in MODULES) + "]", package=PACKAGE))
        cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation",
               "--no-deps", "--find-links", "/opt/wheelhouse", "--target", str(out), str(src)]
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    for m in MODULES:
        assert filecmp.cmp(ref / f"{m}.py", out / f"{m}.py", shallow=False), m
    for f in (ref / PACKAGE).glob("*.py"):
        assert filecmp.cmp(f, out / PACKAGE / f.name, shallow=False), f
    print(f"installed the reference into {out}")
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    sys.exit(main(Path(sys.argv[1]).resolve()))
