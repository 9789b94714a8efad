// Backward pass: gradient of the TLR log-likelihood in (sigma2, range, eta).
//
// No counterpart in the reference (it has no gradient code; its only derivatives are finite
// differences, codes/15_pilot_standard_errors.py:21-31).  With Sigma_t = L L^T the TLR factor of
// the forward pass (ranks frozen), the gradient is
//     dl/dtheta = 1/2 alpha^T dSigma alpha - 1/2 tr(Z dSigma),  alpha = Sigma_t^{-1} y,  Z = Sigma_t^{-1}
// with Z's tiles from the selected-inversion (Takahashi) recurrence on the tile factor, i.e. the
// blocked Cholesky adjoint with the truncations passed through unchanged (oracle:
// oracle/tlr_oracle.py:tlr_loglik_grad).  Reverse step m, with Vp = L_mm^{-T} [V_jm]_{j>m}:
//     Z_im = -sum_{j>m} (Z_ij U_jm) Vp_j^T                       (i > m; Z_ij = Z_ji^T for j > i)
//     Z_mm = L_mm^{-T} L_mm^{-1} - sum_{j>m} (Z_jm^T U_jm) Vp_j^T
// The products Z_ij U_jm are formed once, when Z_ij is, for every m < j, so each dense Z tile is
// read from HBM a fixed number of times.  dSigma tiles are regenerated from the sites inside the
// contraction kernel, never stored.
//
// With C_im = [Z_ij U_jm]_{j>m} (b_i x R_m, contiguous) these are single GEMMs of inner dimension
// R_m = sum_j r_jm; the C blocks are written when Z_ij is formed (column-scattered GEMM output).
// Kernels: a batched FP64 GEMM with optional column scatter, a batched lower-triangular
// inverse (L^{-1} of every diagonal tile), the TLR backward solve for alpha, and the fused dSigma
// generation + contraction.
#include <cooperative_groups.h>

#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace cg = cooperative_groups;

namespace tlr {

// ----------------------------------------------------------------------------------------
// Batched FP64 GEMM  C = alpha op(A) op(B) + beta C on the FP64 tensor cores (mma m8n8k4, exact
// FP64 fused multiply-adds).  64 x 64 output tiles, 256 threads: warp w owns rows 32 (w & 1) and
// columns 16 (w >> 1) of the tile (4 x 2 fragments of 8 x 8).  K advances in slices of 16 through
// shared memory, double-buffered: the next slice is loaded into registers while the tensor cores
// work on the current one.  A job may scatter its output columns: column n then goes to ccol[n]
// (leading rows contiguous) instead of C + n ldc.
constexpr int kDgP = 72;  // slice row pitch in doubles (fragment reads hit every bank pair twice)

__global__ void __launch_bounds__(256, 3) k_dgemm_batched(const GemmJob* TLR_RESTRICT jobs,
                                                      const int* TLR_RESTRICT status, int kind) {
  if (*status != 0) return;
  const GemmJob jb = jobs[blockIdx.z];
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  if (m0 >= jb.M || n0 >= jb.N) return;
  __shared__ double As[2][16][kDgP];
  __shared__ double Bs[2][16][kDgP];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const int wm0 = (warp & 1) * 32, wn0 = (warp >> 1) * 16;
  double ra[4], rb[4];
  // slice k0 -> registers, coalesced along whichever index is contiguous in memory
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      const int kk = jb.transA ? (e & 15) : (e >> 6), mm = jb.transA ? (e >> 4) : (e & 63);
      const int gm = m0 + mm, gk = k0 + kk;
      ra[q] = (gm < jb.M && gk < jb.K) ? (jb.transA ? jb.A[(size_t)gm * jb.lda + gk] : jb.A[(size_t)gk * jb.lda + gm])
                                       : 0.0;
      const int kb = jb.transB ? (e >> 6) : (e & 15), nn = jb.transB ? (e & 63) : (e >> 4);
      const int gn = n0 + nn, gkb = k0 + kb;
      rb[q] = (gn < jb.N && gkb < jb.K) ? (jb.transB ? jb.B[(size_t)gkb * jb.ldb + gn] : jb.B[(size_t)gn * jb.ldb + gkb])
                                        : 0.0;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      const int kk = jb.transA ? (e & 15) : (e >> 6), mm = jb.transA ? (e >> 4) : (e & 63);
      As[buf][kk][mm] = ra[q];
      const int kb = jb.transB ? (e >> 6) : (e & 15), nn = jb.transB ? (e & 63) : (e >> 4);
      Bs[buf][kb][nn] = rb[q];
    }
  };
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  if (jb.K > 0) {
    load(0);
    store(0);
  }
  __syncthreads();
  for (int k0 = 0, buf = 0; k0 < jb.K; k0 += 16, buf ^= 1) {
    const bool more = k0 + 16 < jb.K;
    if (more) load(k0 + 16);
#pragma unroll
    for (int kq = 0; kq < 4; ++kq) {
      double a[4], bv[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[buf][4 * kq + t][wm0 + 8 * i + g];
#pragma unroll
      for (int j = 0; j < 2; ++j) bv[j] = Bs[buf][4 * kq + t][wn0 + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma884(acc[i][j][0], acc[i][j][1], a[i], bv[j]);
    }
    if (more) store(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gn = n0 + wn0 + 8 * j + 2 * t + h;
      if (gn >= jb.N) continue;
      double* cc = jb.ccol ? jb.ccol[gn] : jb.C + (size_t)gn * jb.ldc;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int gm = m0 + wm0 + 8 * i + g;
        if (gm >= jb.M) continue;
        const double v = jb.alpha * acc[i][j][h];
        cc[gm] = (jb.beta == 0.0) ? v : fma(jb.beta, cc[gm], v);
      }
    }
  if (tid == 0) {
    const int mt = min(64, jb.M - m0), nt = min(64, jb.N - n0);
    add_work(status, kind, 2.0 * jb.K * mt * nt, 8.0 * ((double)mt * nt + (double)(mt + nt) * jb.K));
  }
}

int launch_dgemm_batched(const GemmJob* jobs, int njobs, int max_m, int max_n, const int* status, int kind,
                         cudaStream_t s) {
  if (njobs <= 0) return 0;
  dim3 grid((unsigned)((max_n + 63) / 64), (unsigned)((max_m + 63) / 64), (unsigned)njobs);
  k_dgemm_batched<<<grid, 256, 0, s>>>(jobs, status, kind);
  return (int)cudaGetLastError();
}

// ----------------------------------------------------------------------------------------
// Li_k = L_kk^{-1} for every diagonal tile: blocked forward substitution on the identity, one
// CTA per (tile, 32-column block); columns are independent.
__global__ void __launch_bounds__(256) k_tri_inv(const double* TLR_RESTRICT D, double* TLR_RESTRICT Li, int n,
                                                int b, const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const int k = blockIdx.y, cb = blockIdx.x;
  const int bk = min(b, n - k * b);
  const int c0 = cb * 32;
  if (c0 >= bk) return;
  const int cw = min(32, bk - c0);
  const double* L = D + (size_t)k * b * b;
  double* X = Li + (size_t)k * b * b;
  __shared__ double L11[32][33];
  __shared__ double Xp[32][33];
  const int tid = threadIdx.x;
  if (tid == 0 && cb == 0) add_work(status, 13, (double)bk * bk * bk / 3.0, 16.0 * bk * bk);
  // X[:, c0:c0+cw] = identity columns
  for (int c = 0; c < cw; ++c)
    for (int a = tid; a < bk; a += 256) X[(size_t)(c0 + c) * b + a] = (a == c0 + c) ? 1.0 : 0.0;
  __syncthreads();
  for (int p0 = (c0 / 32) * 32; p0 < bk; p0 += 32) {
    const int pw = min(32, bk - p0);
    for (int e = tid; e < 32 * 32; e += 256) {
      const int a = e & 31, c = e >> 5;
      L11[a][c] = (a < pw && c < pw && a >= c) ? L[(size_t)(p0 + c) * b + p0 + a] : 0.0;
    }
    __syncthreads();
    if (tid < cw) {
      double* xc = X + (size_t)(c0 + tid) * b + p0;
      double x[32];
#pragma unroll
      for (int a = 0; a < 32; ++a) x[a] = (a < pw) ? xc[a] : 0.0;
#pragma unroll
      for (int a = 0; a < 32; ++a) {
        if (a < pw) {
          double s = x[a];
#pragma unroll
          for (int c = 0; c < a; ++c) s -= L11[a][c] * x[c];
          x[a] = s / L11[a][a];
        }
      }
#pragma unroll
      for (int a = 0; a < 32; ++a)
        if (a < pw) { xc[a] = x[a]; Xp[a][tid] = x[a]; }
    }
    __syncthreads();
    for (int row = p0 + pw + tid; row < bk; row += 256) {
      double l[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) l[c] = (c < pw) ? L[(size_t)(p0 + c) * b + row] : 0.0;
      for (int q = 0; q < cw; ++q) {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 32; ++c) s = fma(l[c], Xp[c][q], s);
        X[(size_t)(c0 + q) * b + row] -= s;
      }
    }
    __syncthreads();
  }
}

int launch_tri_inv(const double* D, double* Li, int n, int b, int nB, const int* status, cudaStream_t s) {
  dim3 grid((unsigned)((b + 31) / 32), (unsigned)nB);
  k_tri_inv<<<grid, 256, 0, s>>>(D, Li, n, b, status);
  return (int)cudaGetLastError();
}

// ----------------------------------------------------------------------------------------
// Column-block copies (gathers of U / V factors into contiguous panels).
__global__ void k_copy_cols(const CopyJob* TLR_RESTRICT jobs, const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const CopyJob jb = jobs[blockIdx.y];
  const size_t total = (size_t)jb.rows * jb.cols;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e % jb.rows), c = (int)(e / jb.rows);
    jb.dst[(size_t)c * jb.ldd + r] = jb.src[(size_t)c * jb.lds + r];
  }
}

int launch_copy_cols(const CopyJob* jobs, int njobs, const int* status, cudaStream_t s) {
  if (njobs <= 0) return 0;
  dim3 grid(32u, (unsigned)njobs);
  k_copy_cols<<<grid, 256, 0, s>>>(jobs, status);
  return (int)cudaGetLastError();
}

// ----------------------------------------------------------------------------------------
// alpha_m = L_mm^{-T} (z_m - sum_{i>m} V_im (U_im^T alpha_i))   (codes/17_tlr_cholesky_pilot.py:243-256
// restated for one block row).  One cluster of kAC CTAs, three phases separated by the cluster
// barrier: t = [U_im^T alpha_i]_{i>m} (one warp per entry, lanes over rows); rhs = z_m - sum_i
// V_im t_i (rows split across the cluster, four threads per row); alpha_m = L_mm^{-T} rhs (one
// warp per output, lanes over the column of L_mm^{-1}).  t and rhs live in `work` (L2).
constexpr int kAC = 8;

__global__ void __cluster_dims__(kAC, 1, 1) __launch_bounds__(256)
    k_alpha_step(int n, int b, int m, int nB, const double* TLR_RESTRICT U, const double* TLR_RESTRICT V,
                 const int* TLR_RESTRICT rank, int cap, const double* TLR_RESTRICT Li, const double* TLR_RESTRICT z,
                 double* TLR_RESTRICT alpha, double* TLR_RESTRICT work, const int* TLR_RESTRICT status) {
  cg::cluster_group cluster = cg::this_cluster();
  const int g = (int)cluster.block_rank();
  __shared__ int go;
  __shared__ int off[1025];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) go = (g == 0) ? (*status == 0) : 0;
  cluster.sync();
  const int ok = *cluster.map_shared_rank(&go, 0);
  cluster.sync();  // rank 0's shared memory stays valid until every CTA has read it
  if (!ok) return;
  const int bm = min(b, n - m * b);
  double* rhs = work;      // b
  double* tq = work + b;   // sum_{i>m} r_im
  if (tid == 0) {
    int o = 0;
    for (int i = m + 1; i < nB; ++i) {
      off[i - m - 1] = o;
      o += rank[i * (i - 1) / 2 + m];
    }
    off[nB - m - 1] = o;
  }
  __syncthreads();
  const int R = off[nB - m - 1];
  const int nw = kAC * 8, gw = g * 8 + warp;
  for (int e = gw; e < R; e += nw) {
    int lo = 0, hi = nB - m - 1;  // off[lo] <= e < off[lo + 1]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (off[mid] <= e) lo = mid; else hi = mid;
    }
    const int i = m + 1 + lo, q = e - off[lo];
    const int bi = min(b, n - i * b);
    const double* u = U + ((size_t)i * (i - 1) / 2 + m) * b * cap + (size_t)q * b;
    const double* ai = alpha + (size_t)i * b;
    double sacc = 0.0;
    for (int a = lane; a < bi; a += 32) sacc = fma(u[a], ai[a], sacc);
    sacc = warp_sum(sacc);
    if (lane == 0) tq[e] = sacc;
  }
  cluster.sync();
  {
    const int per = (bm + kAC - 1) / kAC;
    const int r0 = g * per, r1 = min(bm, r0 + per);
    const int quarter = tid & 3;
    for (int base = r0; base < r1; base += 64) {  // the same trip count in every thread (shuffles)
      const int a = base + (tid >> 2);
      const bool act = a < r1;
      double sacc = 0.0;
      if (act)
        for (int lo = 0; lo < nB - m - 1; ++lo) {
          const int i = m + 1 + lo, r = off[lo + 1] - off[lo];
          const double* v = V + ((size_t)i * (i - 1) / 2 + m) * b * cap;
          for (int q = quarter; q < r; q += 4) sacc = fma(v[(size_t)q * b + a], tq[off[lo] + q], sacc);
        }
      sacc += __shfl_xor_sync(0xffffffffu, sacc, 1);
      sacc += __shfl_xor_sync(0xffffffffu, sacc, 2);
      if (act && quarter == 0) rhs[a] = z[(size_t)m * b + a] - sacc;
    }
  }
  cluster.sync();
  // alpha_m = L_mm^{-T} rhs: (Li^T rhs)_a = sum_{c >= a} Li[c][a] rhs[c]
  const double* L = Li + (size_t)m * b * b;
  for (int a = gw; a < bm; a += nw) {
    const double* col = L + (size_t)a * b;
    double sacc = 0.0;
    for (int c = a + lane; c < bm; c += 32) sacc = fma(col[c], rhs[c], sacc);
    sacc = warp_sum(sacc);
    if (lane == 0) alpha[(size_t)m * b + a] = sacc;
  }
}

int launch_alpha_step(int n, int b, int m, int nB, const double* U, const double* V, const int* rank, int cap,
                      const double* Li, const double* z, double* alpha, double* work, const int* status,
                      cudaStream_t s) {
  k_alpha_step<<<kAC, 256, 0, s>>>(n, b, m, nB, U, V, rank, cap, Li, z, alpha, work, status);
  return (int)cudaGetLastError();
}

// ----------------------------------------------------------------------------------------
// Contraction of dSigma (regenerated) with Sbar = 1/2 (alpha_i alpha_m^T - Z_im) over the tiles
// (i, m), i >= m, of block column m; weight 2 for off-diagonal tiles.  One CTA per 32 x 32 block;
// partial sums [3] per CTA into part (fixed slots: deterministic final reduction).
__global__ void __launch_bounds__(256) k_dtrace_step(const double* TLR_RESTRICT xy, int n, int b, int m, int nB,
                                                    double sigma2, double inv_range, int nu5, double eta,
                                                    const double* TLR_RESTRICT Zbuf,
                                                    const double* TLR_RESTRICT alpha, double* TLR_RESTRICT part,
                                                    const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const int nb32 = (b + 31) / 32;
  const int per_tile = nb32 * nb32;
  const int i = m + blockIdx.x / per_tile;
  const int blk = blockIdx.x % per_tile;
  const int rb = blk / nb32, cb = blk % nb32;
  double* out = part + (size_t)blockIdx.x * 3;
  const int bi = min(b, n - i * b), bm = min(b, n - m * b);
  const int r0 = rb * 32, c0 = cb * 32;
  const int tid = threadIdx.x;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  if (r0 < bi && c0 < bm) {
    const double* Z = Zbuf + (size_t)(i - m) * b * b;  // Z_im, column-major, ld b
    const double2* p2 = reinterpret_cast<const double2*>(xy);
    const double* ai = alpha + (size_t)i * b;
    const double* am = alpha + (size_t)m * b;
    const int cl = tid & 31, rl = tid >> 5;
    const int c = c0 + cl;
    if (c < bm) {
      const double2 pc = p2[(size_t)m * b + c];
      const double amc = am[c];
      for (int q = 0; q < 4; ++q) {
        const int a = r0 + rl + 8 * q;
        if (a >= bi) continue;
        const double2 pa = p2[(size_t)i * b + a];
        const double dx = pa.x - pc.x, dy = pa.y - pc.y;
        // dk/d sigma2 = k; dk/d range = sigma2 x^2 e^{-x} / range (nu 3/2) or
        // sigma2 x^2 (1 + x) e^{-x} / (3 range) (nu 5/2)
        const double h = sqrt(fmax(dx * dx + dy * dy, 0.0));
        const double x = (nu5 ? kSqrt5 : kSqrt3) * h * inv_range;
        const double e = exp(-x);
        const double sbar = 0.5 * (ai[a] * amc - Z[(size_t)c * b + a]);
        double ds = (nu5 ? 1.0 + x + x * x / 3.0 : 1.0 + x) * e;
        const double dr = nu5 ? sigma2 * x * x * (1.0 + x) / 3.0 * e * inv_range : sigma2 * x * x * e * inv_range;
        double de = 0.0;
        if (i == m && a == c) {
          ds += eta;
          de = sigma2;
        }
        g0 = fma(ds, sbar, g0);
        g1 = fma(dr, sbar, g1);
        g2 = fma(de, sbar, g2);
      }
    }
  }
  __shared__ double red[40];
  const double w = (i == m) ? 1.0 : 2.0;
  g0 = block_sum(g0, red);
  g1 = block_sum(g1, red);
  g2 = block_sum(g2, red);
  if (tid == 0) {
    out[0] = w * g0;
    out[1] = w * g1;
    out[2] = w * g2;
  }
}

int launch_dtrace_step(const double* xy, int n, int b, int m, int nB, double sigma2, double inv_range, int nu5,
                       double eta, const double* Zbuf, const double* alpha, double* part, const int* status,
                       cudaStream_t s) {
  const int nb32 = (b + 31) / 32;
  const int ntile = nB - m;
  k_dtrace_step<<<ntile * nb32 * nb32, 256, 0, s>>>(xy, n, b, m, nB, sigma2, inv_range, nu5, eta, Zbuf, alpha, part,
                                                    status);
  return (int)cudaGetLastError();
}

// final deterministic reduction of the gradient partials: fixed per-thread strides, then a
// fixed-order block reduction
__global__ void __launch_bounds__(1024) k_grad_finish(const double* part, long nparts, double* grad,
                                                     const int* status) {
  __shared__ double red[40];
  if (*status != 0) {
    if (threadIdx.x == 0) grad[0] = grad[1] = grad[2] = 0.0;
    return;
  }
  double g[3] = {0.0, 0.0, 0.0};
  for (long q = threadIdx.x; q < nparts; q += blockDim.x)
    for (int a = 0; a < 3; ++a) g[a] += part[3 * q + a];
  for (int a = 0; a < 3; ++a) {
    const double t = block_sum(g[a], red);
    if (threadIdx.x == 0) grad[a] = t;
  }
}

int launch_grad_finish(const double* part, long nparts, double* grad, const int* status, cudaStream_t s) {
  k_grad_finish<<<1, 1024, 0, s>>>(part, nparts, grad, status);
  return (int)cudaGetLastError();
}

}  // namespace tlr
