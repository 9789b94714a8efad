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


def test_gemm_selftest_rejects_bad_arguments_without_a_gpu():
    """tlr_selftest_gemm checks its arguments before touching a device: unknown precision,
    negative sizes, leading dimensions below the matrix height and missing matrices are errors."""
    lib = _lib.load()
    mixed = _lib.PRECISIONS["mixed"]
    cases = [
        (7, 0, 0, 4, 4, 4, 4, 4, 4),          # precision
        (mixed, 0, 0, -1, 4, 4, 4, 4, 4),     # M < 0
        (mixed, 0, 0, 4, 4, 4, 2, 4, 4),      # lda < M
        (mixed, 1, 0, 4, 4, 8, 4, 8, 4),      # lda < K for op(A) = A^T
        (mixed, 0, 1, 4, 6, 4, 4, 4, 4),      # ldb < N for op(B) = B^T
        (mixed, 0, 0, 4, 4, 4, 4, 4, 3),      # ldc < M
    ]
    for prec, ta, tb, M, N, K, lda, ldb, ldc in cases:
        rc = lib.tlr_selftest_gemm(prec, ta, tb, M, N, K, 1.0, None, lda, None, ldb, 0.0, None, ldc, 0)
        assert rc < 0, (prec, ta, tb, M, N, K, lda, ldb, ldc)
    # sizes are fine but the matrices are missing
    assert lib.tlr_selftest_gemm(mixed, 0, 0, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4, 0) < 0
    assert "NULL" in _lib.last_error()
    # an empty product is a no-op that needs no device
    assert lib.tlr_selftest_gemm(mixed, 0, 0, 0, 4, 4, 1.0, None, 1, None, 4, 0.0, None, 1, 0) == 0
