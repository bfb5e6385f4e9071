"""The C ABI library loads and exports every entry point the header declares
(no compute calls: these run without a GPU)."""

import re
import subprocess

from conftest import ROOT

HEADER = ROOT / "include" / "momwire_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mw_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "mw_fill_z" in names and "mw_zgetrf" in names
    assert len(names) >= 8


def test_library_loads_and_exports_all_symbols():
    from momwire_b200 import _lib

    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True)
    exported = set(re.findall(r"\bT (mw_[a-z0-9_]+)", out.stdout))
    for name in declared_functions():
        assert name in exported, f"{name} declared in the header but not exported"
        assert hasattr(lib, name)
        assert name in _lib.EXPORTED, f"{name} has no ctypes signature"


def test_library_version_and_error_text():
    from momwire_b200 import _lib

    lib = _lib.load()
    assert lib.mw_version() >= 100
    assert isinstance(lib.mw_last_error(), bytes)


def test_invalid_arguments_rejected_without_gpu():
    """Argument validation happens before any CUDA call."""
    from momwire_b200 import _lib

    lib = _lib.load()
    st = lib.mw_zgetrf(-1, None, 1, None, None, None, 0, None, None)
    assert st == _lib.MW_ERR_INVALID
    assert b"bad n/lda" in lib.mw_last_error()
