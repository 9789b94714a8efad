"""ctypes binding of libtlr_b200.so (the C ABI declared in include/tlr_b200.h).

The shared library is built in-tree (``python -m adaptive_tlr_pilots_b200.build`` or
``__graft_entry__.build()``).  There is no fallback: when the library is missing or no CUDA
device is present, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtlr_b200.so")

TLR_RULE_FIXED = 0
TLR_RULE_ADAPTIVE = 1
TLR_RULE_MIXED = 2
PRECISIONS = {"fp64": 0, "mixed": 1}
RANK_MAP = {"rule": 0, "record": 1, "replay": 2}
ERR_RANK_CAP = -2  # TLR_ERR_RANK_CAP: a tile rank exceeded the plan's capacity
ERR_NOMEM = -4  # TLR_ERR_NOMEM: a device allocation failed
DIST_DIAG, DIST_PANEL, DIST_SUMS = 0, 1, 2  # tlr_dist_buffer_doubles: the three exchange buffers

_lib = None

KERNEL_KINDS = ["fill", "gen_offdiag", "sketch", "orth", "project", "resid", "finalize", "diag_build", "potrf",
                "trsm", "recompress", "finish", "bwd_gemm", "tri_inv", "bwd_copy", "alpha", "dtrace", "grad_finish"]


class TlrTileStats(ctypes.Structure):
    _fields_ = [
        ("stored", ctypes.c_longlong),
        ("max_rel", ctypes.c_double),
        ("max_abs", ctypes.c_double),
        ("fro_err", ctypes.c_double),
        ("max_rank", ctypes.c_int),
    ]


class TlrInfo(ctypes.Structure):
    _fields_ = [
        ("completed", ctypes.c_int),
        ("failed_at", ctypes.c_int),
        ("stored_sigma", ctypes.c_longlong),
        ("max_rank_sigma", ctypes.c_int),
        ("stored_factor", ctypes.c_longlong),
        ("mean_rank_factor", ctypes.c_double),
        ("max_rank_factor", ctypes.c_int),
        ("logdet", ctypes.c_double),
        ("quad", ctypes.c_double),
    ]


# name -> (restype, argtypes); every symbol declared in include/tlr_b200.h
SIGNATURES = {
    "tlr_plan_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_void_p]),
    "tlr_plan_destroy": (None, [ctypes.c_void_p]),
    "tlr_morton_order": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "tlr_morton_order_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_void_p]),
    "tlr_set_data": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "tlr_loglik": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_double,
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(TlrInfo),
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "tlr_loglik_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                       ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(TlrInfo),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "tlr_loglik_grad_batch": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_double,
                                             ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_int)]),
    "tlr_loglik_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_double,
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(TlrInfo),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "tlr_factor_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "tlr_factor_matvec": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "tlr_get_diag_tile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "tlr_get_offdiag_tile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "tlr_plan_set_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tlr_plan_rank_map": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tlr_plan_rank_map_size": (ctypes.c_longlong, [ctypes.c_void_p]),
    "tlr_plan_rank_map_io": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                            ctypes.c_longlong, ctypes.c_int]),
    "tlr_factor_storage": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_longlong)]),
    "tlr_truncate_tiles": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                          ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong,
                                          ctypes.POINTER(TlrTileStats), ctypes.POINTER(ctypes.c_int)]),
    "tlr_plan_set_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "tlr_plan_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tlr_plan_set_graphs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tlr_plan_set_partition": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "tlr_dist_buffer_doubles": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "tlr_dist_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                      ctypes.c_double]),
    "tlr_dist_pack_diag": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "tlr_dist_unpack_diag": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "tlr_dist_solve_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tlr_dist_pack_panel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "tlr_dist_unpack_panel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "tlr_dist_update_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tlr_dist_pack_sums": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "tlr_dist_finish": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(TlrInfo), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "tlr_plan_kernel_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int]),
    "tlr_selftest_bounded_wait": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                 ctypes.POINTER(ctypes.c_longlong)]),
    "tlr_selftest_gemm": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                         ctypes.c_int, ctypes.c_int]),
    "tlr_last_error": (ctypes.c_char_p, []),
}


def load(path: str = LIB_PATH):
    """Load the shared library and declare its signatures (no GPU needed)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"the CUDA extension {path} is not built; run adaptive_tlr_pilots_b200.build.build()")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().tlr_last_error().decode(errors="replace")


class TlrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"tlr error {code}: {msg}")
        self.code = code


def check(rc: int) -> int:
    """Raise on rc < 0 (errors); return rc otherwise (0 or the not-PD code k + 1)."""
    if rc < 0:
        raise TlrError(rc, last_error())
    return rc
