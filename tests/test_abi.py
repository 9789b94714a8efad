"""The C-ABI library loads and exports every symbol include/tlr_b200.h declares (no GPU calls)."""
import ctypes
import os
import re

import pytest

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


def test_kernel_switch_validates_and_restores():
    """set_kernel accepts the two smoothness values of the reference (1.5, 2.5) and nothing else,
    in the package and in the oracle."""
    import adaptive_tlr_pilots_b200 as tlr
    from oracle import tlr_oracle as O
    for mod in (tlr, O):
        setter = mod.set_kernel
        with pytest.raises(ValueError):
            setter(2.0)
        setter(2.5)
        setter(1.5)
    assert tlr.get_kernel() == 1.5 and O.NU == 1.5
