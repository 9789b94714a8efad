"""The backward pass's GEMM kernels on their own, through the self-test entry point
tlr_selftest_gemm: C = alpha op(A) op(B) + beta C (column-major) against a float64 product.

FP64 path (FP64 tensor cores): within 1e-13 of sum_k |op(A)_ik| |op(B)_kj|.  Mixed path (split
TF32 on tcgen05, FP32 accumulation): within 2e-6 of that bound, the FP32-class accuracy the
selected-inversion gradient needs.  Shapes cover every transpose pair, ragged tile and slice
edges, K = 0 and 1, odd leading dimensions and an operand that does not start on 16 bytes (the
8-byte copy form of the tensor-core kernel)."""
import itertools

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    from adaptive_tlr_pilots_b200 import _lib
    return torch, _lib, _lib.load()


def _operand(torch, rows, cols, ld, shift, g):
    """Column-major rows x cols matrix with leading dimension ld, starting `shift` doubles into a
    fresh buffer; returns (pointer, view as a rows x cols tensor)."""
    buf = torch.randn(shift + cols * ld, dtype=torch.float64, generator=g).cuda()
    stor = buf[shift:].view(cols, ld)
    return buf, stor.data_ptr(), stor[:, :rows].T


def _run(env, precision, transA, transB, M, N, K, alpha, beta, pad=0, shift=0, seed=0):
    torch, _lib, lib = env
    g = torch.Generator().manual_seed(seed)
    am, ak = (K, M) if transA else (M, K)     # stored A is am x ak; op(A) = A or A^T
    bm, bk = (N, K) if transB else (K, N)
    lda, ldb, ldc = max(1, am) + pad, max(1, bm) + pad, max(1, M) + pad
    keep = []
    bufA, pA, A = _operand(torch, am, ak, lda, shift, g)
    bufB, pB, B = _operand(torch, bm, bk, ldb, 0, g)
    bufC, pC, C = _operand(torch, M, N, ldc, 0, g)
    keep += [bufA, bufB, bufC]
    opA = A.T if transA else A
    opB = B.T if transB else B
    ref = alpha * (opA.cpu() @ opB.cpu()) + beta * C.cpu()
    bound = (opA.abs().cpu() @ opB.abs().cpu()) * abs(alpha) + abs(beta) * C.abs().cpu()
    torch.cuda.synchronize()
    rc = lib.tlr_selftest_gemm(_lib.PRECISIONS[precision], transA, transB, M, N, K, alpha, pA, lda, pB, ldb, beta,
                               pC, ldc, 0)
    assert rc == 0, (rc, _lib.last_error())
    err = ((C.cpu() - ref).abs() / bound.clamp_min(1e-300)).max().item() if M * N else 0.0
    return err


SHAPES = [(500, 500, 320), (128, 128, 16), (129, 127, 17), (1, 1, 1), (37, 300, 5), (260, 45, 0), (300, 200, 97),
          (64, 513, 48)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-6)])
@pytest.mark.parametrize("transA,transB", list(itertools.product((0, 1), (0, 1))))
def test_gemm_shapes(env, precision, tol, transA, transB):
    for i, (M, N, K) in enumerate(SHAPES):
        err = _run(env, precision, transA, transB, M, N, K, 1.0, 0.0, seed=i)
        assert err <= tol, (precision, transA, transB, M, N, K, err)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-6)])
def test_gemm_alpha_beta_and_layouts(env, precision, tol):
    cases = [  # (transA, transB, M, N, K, alpha, beta, pad, shift)
        (0, 1, 250, 300, 100, -1.0, 1.0, 0, 0),
        (1, 0, 130, 140, 70, 0.5, -2.0, 1, 0),      # odd leading dimensions: 8-byte copies
        (0, 0, 200, 90, 33, 1.0, 0.0, 0, 1),        # A one double off 16 bytes: 8-byte copies
        (1, 1, 77, 260, 250, 2.0, 0.25, 3, 1),
    ]
    for i, (ta, tb, M, N, K, al, be, pad, shift) in enumerate(cases):
        err = _run(env, precision, ta, tb, M, N, K, al, be, pad=pad, shift=shift, seed=100 + i)
        assert err <= tol, (precision, ta, tb, M, N, K, al, be, pad, shift, err)


def test_gemm_rejects_bad_arguments(env):
    torch, _lib, lib = env
    assert lib.tlr_selftest_gemm(7, 0, 0, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4, 0) < 0
    assert lib.tlr_selftest_gemm(_lib.PRECISIONS["mixed"], 0, 0, 4, 4, 4, 1.0, None, 2, None, 4, 0.0, None, 4, 0) < 0
