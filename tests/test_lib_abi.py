"""The C-ABI library loads and exports what include/eemd_b200.h declares.

Only host-side entry points are called here (no GPU work): version, strerror,
default parameters, workspace sizing and argument validation.
"""
import ctypes
import re
from pathlib import Path

import pytest

from eemd4cuda_b200 import _lib as L

HEADER = Path(__file__).resolve().parents[1] / "include" / "eemd_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(eemd_[a-z_]+)\s*\(", text)))


def test_header_lists_the_bound_symbols():
    assert declared_functions() == sorted(L.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(L.lib_path()))
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_checked_build_exports_too():
    p = L.LIB_DIR / "libeemd_b200_checked.so"
    lib = ctypes.CDLL(str(p))
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_header_constants_match_the_binding():
    """Every status code, mode constant and the static scratch size that the
    ctypes binding hard-codes equal the header's #defines."""
    text = HEADER.read_text()
    defs = {}
    for name, val in re.findall(r"#define\s+(EEMD_[A-Z0-9_]+)\s+(\S[^/\n]*)", text):
        defs[name] = val.strip()
    m = re.fullmatch(r"\((\d+)u \* (\d+)u \* (\d+)u\)", defs["EEMD_STATIC_SCRATCH_BYTES"])
    assert m, defs["EEMD_STATIC_SCRATCH_BYTES"]
    assert int(m[1]) * int(m[2]) * int(m[3]) == L.STATIC_SCRATCH_BYTES
    checked = 0
    for name, val in defs.items():
        if hasattr(L, name) and re.fullmatch(r"-?\d+", val):
            assert getattr(L, name) == int(val), name
            checked += 1
    assert int(defs["EEMD_ABI_VERSION"]) == L.ABI_VERSION
    assert checked >= 19


def test_version_and_strerror():
    lib = L.load()
    assert lib.eemd_version() == L.ABI_VERSION
    assert L.strerror(0) == "ok"
    assert "workspace" in L.strerror(L.EEMD_E_NOMEM)
    assert "watchdog" in L.strerror(L.EEMD_E_TIMEOUT)


def test_struct_layout():
    assert ctypes.sizeof(L.EemdParams) == 96
    assert L.EemdParams.cta_warps.offset == 88
    assert L.EemdParams.watchdog.offset == 72
    p = L.default_params()
    assert p.dtype == L.EEMD_F64 and p.max_sifts == 50 and p.min_extrema == 4
    assert abs(p.tau - 0.25) < 1e-15 and p.rules == L.EEMD_RULES_REF


def test_workspace_size_scales():
    p = L.default_params()
    p.max_imf = 8
    a = L.workspace_size(p, [48000], 1, False)
    b = L.workspace_size(p, [48000], 10, False)
    c = L.workspace_size(p, [48000], 10, True)
    assert 9 * a < b < 11 * a + 4096
    assert c < b  # external IMF buffer is not carved from the workspace
    p.dtype = L.EEMD_F32
    assert L.workspace_size(p, [48000], 10, False) < b


@pytest.mark.parametrize("field,value", [("dtype", 7), ("max_sifts", 0), ("max_imf", 0),
                                         ("end_mode", 5), ("rules", 9), ("tile", 300),
                                         ("noise_mode", 11), ("tile", 2048),
                                         ("cluster_size", 17), ("knots_per_block", 8192),
                                         ("halo", 300)])
def test_bad_params_rejected(field, value):
    p = L.default_params()
    setattr(p, field, value)
    with pytest.raises(ValueError):
        L.workspace_size(p, [1000], 1, False)


def test_exact_float32_not_supported():
    p = L.default_params()
    p.dtype = L.EEMD_F32
    p.exact = 1
    with pytest.raises(L.EngineError) as ei:
        L.workspace_size(p, [1000], 1, False)
    assert ei.value.status == L.EEMD_E_NOTSUP


def test_short_signal_rejected():
    p = L.default_params()
    with pytest.raises(ValueError):
        L.workspace_size(p, [2], 1, False)


def test_run_rejects_small_workspace_without_touching_the_device():
    """eemd_run validates sizes on the host before any CUDA call."""
    lib = L.load()
    p = L.default_params()
    la = L.lengths_array([1000])
    need = L.workspace_size(p, [1000], 1, False)
    rc = lib.eemd_run(ctypes.byref(p), ctypes.c_void_p(16), la, 1, 0, 1, None, None, None, None,
                      None, None, None, None, None, None, ctypes.c_void_p(16), need - 1, None)
    assert rc == L.EEMD_E_NOMEM
    rc = lib.eemd_run(ctypes.byref(p), None, la, 1, 0, 1, None, None, None, None,
                      None, None, None, None, None, None, ctypes.c_void_p(16), need, None)
    assert rc == L.EEMD_E_BADARG
    p.noise_mode = L.EEMD_NOISE_INJECTED
    rc = lib.eemd_run(ctypes.byref(p), ctypes.c_void_p(16), la, 1, 0, 1, None, None, None, None,
                      None, None, None, None, None, None, ctypes.c_void_p(16), need, None)
    assert rc == L.EEMD_E_BADARG


@pytest.mark.parametrize("header,module", [("eemd_surrogate.h", "_sg"), ("eemd_spectra.h", "_sp")])
def test_other_libraries_export_their_headers(header, module):
    import importlib
    mod = importlib.import_module(f"eemd4cuda_b200.{module}")
    text = re.sub(r"/\*.*?\*/", "", (HEADER.parent / header).read_text(), flags=re.S)
    declared = sorted(set(re.findall(r"\b(eemd_[a-z_]+)\s*\(", text)))
    assert declared == sorted(mod.EXPORTS)
    lib = ctypes.CDLL(str(mod.lib_path()))
    for name in declared:
        assert hasattr(lib, name), name


def test_flac_library_exports_its_header():
    text = re.sub(r"/\*.*?\*/", "", (HEADER.parent / "eemd_flac.h").read_text(), flags=re.S)
    declared = sorted(set(re.findall(r"\b(eemd_[a-z_]+)\s*\(", text)))
    assert declared == ["eemd_flac_decode", "eemd_flac_info", "eemd_flac_strerror"]
    lib = ctypes.CDLL(str(HEADER.parents[1] / "eemd4cuda_b200" / "lib" / "libeemd_flac.so"))
    for name in declared:
        assert hasattr(lib, name), name


def test_stft_shape_matches_the_reference_frame_count():
    from eemd4cuda_b200 import _sp
    # scipy.signal.stft(boundary='zeros', padded=False): N + 2*(nperseg//2) samples, hop nperseg - noverlap
    for N, nper, nov in [(48000, 4096, 2048), (3000, 256, 128), (4097, 512, 384), (2048, 2048, 1024)]:
        F, T = _sp.stft_shape(N, nper, nov)
        assert F == nper // 2 + 1
        assert T == (N + 2 * (nper // 2) - nov) // (nper - nov)
    with pytest.raises(_sp.SpectraError):
        _sp.stft_shape(100, 64, 64)


def test_headers_are_plain_c99(tmp_path):
    """Every public header compiles as ISO C99 (no C++, no CUDA types), so
    cgo, cffi or any C toolchain can bind the libraries."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    inc = HEADER.parent
    src = tmp_path / "abi.c"
    src.write_text("".join(f'#include "{h.name}"\n' for h in sorted(inc.glob("*.h")))
                   + "int main(void) { return 0; }\n")
    r = subprocess.run([gcc, "-std=c99", "-pedantic-errors", "-Wall", "-Werror", "-fsyntax-only",
                        "-I", str(inc), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_program_links_and_calls_host_entry_points(tmp_path):
    """A plain C program links against libeemd_b200.so through the header and
    calls its host-only entry points (no GPU work): defaults, version,
    workspace sizing, argument refusal and status strings."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    lib = Path(L.lib_path())
    src = tmp_path / "host.c"
    src.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "eemd_b200.h"
int main(void) {
    eemd_params p;
    eemd_default_params(&p);
    if (p.dtype != EEMD_F64 || p.max_sifts != 50 || p.tau != 0.25) return 1;
    if (eemd_version() <= 0) return 2;
    int64_t n[2] = {48000, 1000};
    size_t ws = 0;
    if (eemd_workspace_size(&p, n, 2, 10, 0, &ws) != EEMD_OK || ws == 0) return 3;
    p.max_sifts = 0;
    if (eemd_workspace_size(&p, n, 2, 10, 0, &ws) != EEMD_E_BADARG) return 4;
    if (strlen(eemd_strerror(EEMD_E_BADARG)) == 0) return 5;
    printf("%zu\n", ws);
    return 0;
}
''')
    exe = tmp_path / "host"
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", str(HEADER.parent), str(src),
                        "-L", str(lib.parent), "-l:" + lib.name, "-Wl,-rpath," + str(lib.parent),
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, (run.returncode, run.stderr)
    p = L.default_params()
    assert int(run.stdout) == L.workspace_size(p, [48000, 1000], 10, False)
