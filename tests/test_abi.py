"""The C ABI library loads and exports every symbol include/*.h declares (CPU)."""
import re
from pathlib import Path

import pytest

from swiftimpute_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(si_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ["si_ctx_create", "si_panel_upload_u8", "si_pbwt_build", "si_select_states", "si_impute",
                 "si_impute_device", "si_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = N.load()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    bound = {name for name, _, _ in N.SIGNATURES}
    assert declared_symbols() <= bound


def test_abi_version_and_status_strings():
    lib = N.load()
    assert lib.si_abi_version() == 1
    assert lib.si_status_string(0) == b"ok"
    assert lib.si_status_string(7) == b"HBM budget exceeded"


def test_params_default_matches_reference_hmm_defaults():
    p = N.default_params()
    # HMMParameters defaults, core/types.hpp:84-89
    assert (p.num_states, p.ne, p.rho_rate, p.theta) == (8, 10000, 4.0, pytest.approx(0.001))
    assert p.transition_mode == N.TRANS_MATRIX0 and p.sampling == N.SAMPLE_ARGMAX


def test_no_fallback_when_library_missing(monkeypatch, tmp_path):
    monkeypatch.setattr(N, "LIB_PATH", tmp_path / "missing.so")
    monkeypatch.setattr(N, "_lib", None)
    with pytest.raises(N.NativeLibraryError):
        N.load()


MIRRORS = {"si_impute_params": "ImputeParams", "si_region": "Region", "si_job": "Job",
           "si_serve_config": "ServeConfig", "si_request": "Request", "si_serve_statistics": "ServeStatistics"}


def test_header_is_c99_and_ctypes_layouts_match(tmp_path):
    """A cgo / JNI / ctypes binder parses the header as C: it must compile as
    C99, and every struct's size and field offsets seen by the C compiler must
    equal the Python mirrors' (a mismatch would corrupt arguments silently)."""
    import ctypes
    import subprocess
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "swiftimpute_b200.h"', "int main(void) {"]
    for c_name, py_name in MIRRORS.items():
        cls = getattr(N, py_name)
        lines.append(f'printf("{c_name} size %zu\\n", sizeof({c_name}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{c_name} {field} %zu\\n", offsetof({c_name}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", str(ROOT / "include"), str(src),
                    "-o", str(exe)], check=True)
    seen = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        struct, key, value = line.split()
        seen[(struct, key)] = int(value)
    for c_name, py_name in MIRRORS.items():
        cls = getattr(N, py_name)
        assert seen[(c_name, "size")] == ctypes.sizeof(cls), c_name
        for field, _ in cls._fields_:
            assert seen[(c_name, field)] == getattr(cls, field).offset, f"{c_name}.{field}"
