"""The C-ABI library loads and exports every symbol include/clast_gpu.h
declares (no device calls)."""
import ctypes
import os
import re

from clast_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "clast_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(clast_[a-z_0-9]+)\s*\(", text)))


def test_header_symbols_exported():
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = declared_functions()
    assert "clast_search" in names and "clast_index_build" in names
    for n in names:
        assert hasattr(lib, n), n


def test_binding_covers_header():
    assert set(declared_functions()) <= set(_native.SIGNATURES)


def test_binding_loads():
    lib = _native.load()
    assert lib.clast_last_error(None) == b"null context"
