"""The C-ABI library loads and exports every symbol include/tlr_b200.h declares (no GPU calls)."""
import ctypes
import os
import re

from adaptive_tlr_pilots_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "tlr_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(tlr_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_functions():
    names = declared_functions()
    assert "tlr_loglik" in names and "tlr_plan_create" in names and len(names) >= 9


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_bindings_cover_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)
    _lib.load()
