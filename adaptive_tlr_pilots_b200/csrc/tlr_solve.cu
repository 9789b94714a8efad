// Solves and products with the TLR factor left in a plan by an evaluation (kriging prediction,
// simulation of fields without a dense factor).
//
// Reference: codes/17_tlr_cholesky_pilot.py:218-227 (tlr_matvec_L, Y = L Z), 230-240
// (tlr_forward, L X = B) and 243-256 (tlr_backward, L^T X = Z), each for m right-hand sides.
// Right-looking block order: after the diagonal block X_k is solved, its contribution leaves
// every other block row at once (one CTA per block row and 32-column chunk), so a solve is 2 nB
// launches whatever m.  Column-major N x m operands (ld = N), in place.
#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace tlr {

namespace {

__device__ __forceinline__ int stidx(int i, int j) { return i * (i - 1) / 2 + j; }

constexpr int kSC = 16;  // columns per CTA in the diagonal solves

// X_k <- L_kk^{-1} X_k (trans 0) or L_kk^{-T} X_k (trans 1), kSC columns per CTA staged in shared
// memory, panels of 32 rows.
__global__ void __launch_bounds__(256) k_tri_solve(const double* TLR_RESTRICT D, int n, int b, int k,
                                                  double* TLR_RESTRICT X, int ldx, int m, int trans) {
  const int bk = min(b, n - k * b);
  const int c0 = blockIdx.x * kSC, nc = min(kSC, m - c0);
  const double* L = D + (size_t)k * b * b;
  extern __shared__ double xs[];  // bk x (kSC + 1)
  __shared__ double L11[32][33];
  __shared__ double dinv[32];
  const int tid = threadIdx.x;
  const int ld = kSC + 1;
  for (int e = tid; e < bk * kSC; e += 256) {
    const int r = e % bk, c = e / bk;
    xs[(size_t)r * ld + c] = c < nc ? X[(size_t)(c0 + c) * ldx + (size_t)k * b + r] : 0.0;
  }
  __syncthreads();
  const int np = (bk + 31) / 32;
  for (int pi = 0; pi < np; ++pi) {
    const int p = trans ? np - 1 - pi : pi;
    const int p0 = p * 32, pw = min(32, bk - p0);
    for (int e = tid; e < 32 * 32; e += 256) {
      const int a = e & 31, c = e >> 5;
      L11[a][c] = (a < pw && c < pw && a >= c) ? L[(size_t)(p0 + c) * b + p0 + a] : 0.0;
    }
    if (tid < 32) dinv[tid] = tid < pw ? 1.0 / L[(size_t)(p0 + tid) * b + p0 + tid] : 0.0;
    if (trans) {
      // x_p -= L[below, p]^T x_below, one thread per (panel row q, column c) pair
      for (int e = tid; e < 32 * kSC; e += 256) {
        const int q = e / kSC, c = e % kSC;
        if (q < pw) {
          const double* lc = L + (size_t)(p0 + q) * b;
          double acc = 0.0;
          for (int r = p0 + pw; r < bk; ++r) acc = fma(lc[r], xs[(size_t)r * ld + c], acc);
          xs[(size_t)(p0 + q) * ld + c] -= acc;
        }
      }
    }
    __syncthreads();
    if (tid < kSC) {  // the 32 x 32 diagonal block, one thread per column
      const int c = tid;
      if (!trans) {
        for (int a = 0; a < pw; ++a) {
          double s = xs[(size_t)(p0 + a) * ld + c];
          for (int q = 0; q < a; ++q) s = fma(-L11[a][q], xs[(size_t)(p0 + q) * ld + c], s);
          xs[(size_t)(p0 + a) * ld + c] = s * dinv[a];
        }
      } else {
        for (int a = pw - 1; a >= 0; --a) {
          double s = xs[(size_t)(p0 + a) * ld + c];
          for (int q = a + 1; q < pw; ++q) s = fma(-L11[q][a], xs[(size_t)(p0 + q) * ld + c], s);
          xs[(size_t)(p0 + a) * ld + c] = s * dinv[a];
        }
      }
    }
    __syncthreads();
    if (!trans) {  // rows below the panel: x_below -= L[below, p] x_p
      for (int e = tid; e < (bk - p0 - pw) * kSC; e += 256) {
        const int r = p0 + pw + e / kSC, c = e % kSC;
        double acc = 0.0;
        for (int q = 0; q < pw; ++q) acc = fma(L[(size_t)(p0 + q) * b + r], xs[(size_t)(p0 + q) * ld + c], acc);
        xs[(size_t)r * ld + c] -= acc;
      }
      __syncthreads();
    }
  }
  for (int e = tid; e < bk * nc; e += 256) {
    const int r = e % bk, c = e / bk;
    X[(size_t)(c0 + c) * ldx + (size_t)k * b + r] = xs[(size_t)r * ld + c];
  }
}

// trans 0: X_i -= U_ik (V_ik^T X_k) for i > k;  trans 1: X_j -= V_kj (U_kj^T X_k) for j < k.
// One CTA per (block row, 32-column chunk).
__global__ void __launch_bounds__(256) k_solve_update(const double* TLR_RESTRICT U, const double* TLR_RESTRICT V,
                                                     const int* TLR_RESTRICT rank, int cap, int n, int b, int k,
                                                     double* TLR_RESTRICT X, int ldx, int m, int trans) {
  const int o = trans ? (int)blockIdx.x : k + 1 + (int)blockIdx.x;  // the block row updated
  const int t = trans ? stidx(k, o) : stidx(o, k);
  const int r = rank[t];
  if (r == 0) return;
  const int c0 = blockIdx.y * 32, nc = min(32, m - c0);
  const int bk = min(b, n - k * b), bo = min(b, n - o * b);
  // project with the factor on the k side, expand with the one on the other side
  const double* P = (trans ? U : V) + (size_t)t * b * cap;
  const double* E = (trans ? V : U) + (size_t)t * b * cap;
  __shared__ double T[64][33];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int q0 = 0; q0 < r; q0 += 64) {
    const int rq = min(64, r - q0);
    __syncthreads();
    for (int e = warp; e < rq * nc; e += 8) {
      const int q = e % rq, c = e / rq;
      const double* pc = P + (size_t)(q0 + q) * b;
      const double* xc = X + (size_t)(c0 + c) * ldx + (size_t)k * b;
      double acc = 0.0;
      for (int a = lane; a < bk; a += 32) acc = fma(pc[a], xc[a], acc);
      acc = warp_sum(acc);
      if (lane == 0) T[q][c] = acc;
    }
    __syncthreads();
    for (int e = tid; e < bo * nc; e += 256) {
      const int a = e % bo, c = e / bo;
      double acc = 0.0;
      for (int q = 0; q < rq; ++q) acc = fma(E[(size_t)(q0 + q) * b + a], T[q][c], acc);
      X[(size_t)(c0 + c) * ldx + (size_t)o * b + a] -= acc;
    }
  }
}

// Y_k = L_kk Z_k + sum_{j<k} U_kj (V_kj^T Z_j); one CTA per (block row, 32-column chunk).
__global__ void __launch_bounds__(256) k_matvec_L(const double* TLR_RESTRICT D, const double* TLR_RESTRICT U,
                                                 const double* TLR_RESTRICT V, const int* TLR_RESTRICT rank,
                                                 int cap, int n, int b, const double* TLR_RESTRICT Z, int ldz,
                                                 double* TLR_RESTRICT Y, int ldy, int m) {
  const int k = blockIdx.x;
  const int c0 = blockIdx.y * 32, nc = min(32, m - c0);
  const int bk = min(b, n - k * b);
  const double* L = D + (size_t)k * b * b;
  __shared__ double T[64][33];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < bk * nc; e += 256) {
    const int a = e % bk, c = e / bk;
    const double* zc = Z + (size_t)(c0 + c) * ldz + (size_t)k * b;
    double acc = 0.0;
    for (int q = 0; q <= a; ++q) acc = fma(L[(size_t)q * b + a], zc[q], acc);
    Y[(size_t)(c0 + c) * ldy + (size_t)k * b + a] = acc;
  }
  for (int j = 0; j < k; ++j) {
    const int t = stidx(k, j);
    const int r = rank[t];
    if (r == 0) continue;
    const int bj = min(b, n - j * b);
    const double* Ut = U + (size_t)t * b * cap;
    const double* Vt = V + (size_t)t * b * cap;
    for (int q0 = 0; q0 < r; q0 += 64) {
      const int rq = min(64, r - q0);
      __syncthreads();
      for (int e = warp; e < rq * nc; e += 8) {
        const int q = e % rq, c = e / rq;
        const double* vc = Vt + (size_t)(q0 + q) * b;
        const double* zc = Z + (size_t)(c0 + c) * ldz + (size_t)j * b;
        double acc = 0.0;
        for (int a = lane; a < bj; a += 32) acc = fma(vc[a], zc[a], acc);
        acc = warp_sum(acc);
        if (lane == 0) T[q][c] = acc;
      }
      __syncthreads();
      for (int e = tid; e < bk * nc; e += 256) {
        const int a = e % bk, c = e / bk;
        double acc = 0.0;
        for (int q = 0; q < rq; ++q) acc = fma(Ut[(size_t)(q0 + q) * b + a], T[q][c], acc);
        Y[(size_t)(c0 + c) * ldy + (size_t)k * b + a] += acc;
      }
    }
  }
}

}  // namespace

int launch_factor_solve(const double* D, const double* U, const double* V, const int* rank, int cap, int n, int b,
                        int nB, double* X, int m, int trans, cudaStream_t s) {
  const size_t sm = (size_t)b * (kSC + 1) * sizeof(double);
  cudaFuncSetAttribute(k_tri_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const dim3 gu(1, (m + 31) / 32);
  for (int q = 0; q < nB; ++q) {
    const int k = trans ? nB - 1 - q : q;
    k_tri_solve<<<(m + kSC - 1) / kSC, 256, sm, s>>>(D, n, b, k, X, n, m, trans);
    const int rows = trans ? k : nB - k - 1;
    if (rows > 0) {
      const dim3 g(rows, gu.y);
      k_solve_update<<<g, 256, 0, s>>>(U, V, rank, cap, n, b, k, X, n, m, trans);
    }
  }
  return (int)cudaGetLastError();
}

int launch_factor_matvec(const double* D, const double* U, const double* V, const int* rank, int cap, int n, int b,
                         int nB, const double* Z, double* Y, int m, cudaStream_t s) {
  const dim3 g(nB, (m + 31) / 32);
  k_matvec_L<<<g, 256, 0, s>>>(D, U, V, rank, cap, n, b, Z, n, Y, n, m);
  return (int)cudaGetLastError();
}

}  // namespace tlr
