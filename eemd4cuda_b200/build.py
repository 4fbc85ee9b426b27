"""Build the sm_100a engine library in-tree.

    python -m eemd4cuda_b200.build            # release + checked libraries

Outputs (git-ignored, shipped next to the sources):
    eemd4cuda_b200/lib/libeemd_b200.so          release build
    eemd4cuda_b200/lib/libeemd_b200_checked.so  -DEEMD_CHECKED: every staged
        index is range-checked on the device and a violation is reported as an
        error status instead of an out-of-bounds access
    eemd4cuda_b200/lib/libeemd_b200_trace.so    -DEEMD_TRACE: the persistent
        kernel sums clock64() cycles per phase into the workspace header
        (eemd4cuda_b200.trace reads them)
    eemd4cuda_b200/lib/libeemd_surrogate.so     the learned surrogate's kernels
    eemd4cuda_b200/lib/libeemd_spectra.so       Hilbert IF / STFT of the IMFs (its own FFT)
    eemd4cuda_b200/lib/libeemd_flac.so          FLAC decoder (host C, gcc)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-shared",
    "-I", str(INCLUDE),
]
SOURCES = ["eemd_engine.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the sm_100a engine cannot be built")


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps)


SG_SOURCES = ["surrogate.cu"]
SP_SOURCES = ["spectra.cu"]


def _cuda_lib_dir() -> str:
    return str(Path(nvcc()).resolve().parents[1] / "lib64")


def build(force: bool = False, verbose: bool = False) -> list[Path]:
    LIB.mkdir(exist_ok=True)
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    outs = []
    # the surrogate's kernels (a library of their own; default float contraction)
    out = LIB / "libeemd_surrogate.so"
    outs.append(out)
    sg_deps = [CSRC / s for s in SG_SOURCES] + [INCLUDE / "eemd_surrogate.h"]
    if force or _stale(out, sg_deps):
        tmp = out.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               "-I", str(INCLUDE), "-o", str(tmp), *[str(CSRC / s) for s in SG_SOURCES]]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, out)
    # the spectra stage (its own FFT; no FFT library)
    out = LIB / "libeemd_spectra.so"
    outs.append(out)
    sp_deps = [CSRC / s for s in SP_SOURCES] + [INCLUDE / "eemd_spectra.h"]
    if force or _stale(out, sp_deps):
        tmp = out.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               "-I", str(INCLUDE), "-o", str(tmp), *[str(CSRC / s) for s in SP_SOURCES]]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, out)
    # the FLAC decoder (host code)
    out = LIB / "libeemd_flac.so"
    outs.append(out)
    fl_deps = [CSRC / "flac_decode.c", INCLUDE / "eemd_flac.h"]
    if force or _stale(out, fl_deps):
        tmp = out.with_suffix(".so.tmp")
        cmd = [os.environ.get("CC", "gcc"), "-std=c99", "-O2", "-Wall", "-fPIC", "-shared", "-I", str(INCLUDE),
               "-o", str(tmp), str(CSRC / "flac_decode.c")]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, out)
    for name, extra in (("libeemd_b200.so", []), ("libeemd_b200_checked.so", ["-DEEMD_CHECKED"]),
                        ("libeemd_b200_trace.so", ["-DEEMD_TRACE"])):
        out = LIB / name
        outs.append(out)
        if not force and not _stale(out, deps):
            continue
        tmp = out.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-o", str(tmp), *[str(CSRC / s) for s in SOURCES]]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, out)
    return outs


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv, verbose=True):
        print(p)
