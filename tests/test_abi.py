"""The C-ABI library builds, loads without a GPU and exports every declared entry point."""
import re
from pathlib import Path

from conftest import REPO


def declared_symbols():
    text = (REPO / "include" / "ama.h").read_text()
    return sorted(set(re.findall(r"AMA_API\s+[\w\s\*]+?\b(ama_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from amaterasu_b200 import _lib
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert lib.ama_version() >= 100


def test_errors_surface_without_gpu():
    import ctypes as ct
    from amaterasu_b200 import _lib
    lib = _lib.load()
    rc = lib.ama_engine_create(None, None)
    assert rc == _lib.AMA_ERR_ARG
    assert b"null" in lib.ama_last_error()
