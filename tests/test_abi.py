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
