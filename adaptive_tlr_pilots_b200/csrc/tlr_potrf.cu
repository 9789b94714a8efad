// Cholesky of one diagonal tile spread over several SMs, then the tile's forward-solve block.
//
// Reference: codes/17_tlr_cholesky_pilot.py:171-177 (scipy.linalg.cholesky of A_kk; a pivot that
// is not positive stops the factorization, failed_at = k) and 230-240 (z_k = L_kk^{-1} rhs_k).
//
// One cooperative grid of G CTAs works on the column-major lower triangle of A_kk (L2-resident),
// right-looking in panels of 32 columns:
//   every CTA factors the 32 x 32 diagonal block redundantly in shared memory (identical inputs,
//   identical results, so a non-positive pivot is seen by all CTAs at the same point and they all
//   leave together); the rows below the block are split across CTAs (X = A21 L11^{-T});
//   grid sync; the lower-triangular 32 x 32 blocks of the trailing matrix are split across CTAs
//   (A22 -= X X^T); grid sync.
// The forward solve is fused: each CTA solves z_p = L11^{-1} rhs_p for the panel's rows and
// subtracts X z_p from the right-hand side rows it owns; CTA 0 writes z_k, log det and z_k^T z_k.
#include <cooperative_groups.h>

#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace cg = cooperative_groups;

namespace tlr {

constexpr int kPB = 32;  // panel width

__global__ void __launch_bounds__(256) k_potrf_coop(double* TLR_RESTRICT D, int n, int b, int k,
                                                   double* TLR_RESTRICT rhs, double* TLR_RESTRICT z,
                                                   double* TLR_RESTRICT ldpart, double* TLR_RESTRICT qpart,
                                                   int* TLR_RESTRICT status) {
  cg::grid_group grid = cg::this_grid();
  if (*status != 0) return;  // every CTA reads the same value: all leave together
  const int bk = min(b, n - k * b);
  double* A = D + (size_t)k * b * b;
  double* rk = rhs + (size_t)k * b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = gridDim.x, g = blockIdx.x;
  __shared__ double L11[kPB][kPB + 1];
  __shared__ double Pa[kPB][kPB + 1];
  __shared__ double Pc[kPB][kPB + 1];
  __shared__ double zp[kPB];
  __shared__ int fail;
  __shared__ double logdet_acc, quad_acc;
  if (tid == 0) {
    fail = 0;
    logdet_acc = 0.0;
    quad_acc = 0.0;
    if (g == 0) add_work(status, 8, (double)bk * bk * bk / 3.0 + (double)bk * bk, 8.0 * bk * bk);
  }
  for (int p0 = 0; p0 < bk; p0 += kPB) {
    const int pw = min(kPB, bk - p0);
    const int m = bk - p0 - pw;
    __syncthreads();
    if (warp == 0) {
      // Cholesky of the pw x pw diagonal block, lane = row, the row in registers
      double row[kPB];
#pragma unroll
      for (int j = 0; j < kPB; ++j)
        row[j] = (lane < pw && j <= lane) ? A[(size_t)(p0 + j) * b + p0 + lane] : 0.0;
      int bad = 0;
#pragma unroll
      for (int c = 0; c < kPB; ++c) {
        if (c < pw && !bad) {
          const double d = __shfl_sync(0xffffffffu, row[c], c);
          if (!(d > 0.0)) {
            bad = 1;  // the same pivot in every lane: the whole warp stops here
          } else {
            const double sd = sqrt(d);
            if (lane == c) row[c] = sd;
            if (lane > c) row[c] /= sd;
#pragma unroll
            for (int j = c + 1; j < kPB; ++j) {
              const double ljc = __shfl_sync(0xffffffffu, row[c], j);
              if (lane >= j) row[j] = fma(-row[c], ljc, row[j]);
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < kPB; ++j) L11[lane][j] = (j <= lane) ? row[j] : 0.0;
      __syncwarp();
      if (lane == 0) {
        fail = bad;
        if (!bad) {
          double s = logdet_acc;
          for (int c = 0; c < pw; ++c) s += log(L11[c][c]);
          logdet_acc = s;
        }
      }
      // z_p = L11^{-1} rhs_p (the forward solve of this block, fused)
      if (!bad) {
        double v = (lane < pw) ? rk[p0 + lane] : 0.0;
        for (int c = 0; c < pw; ++c) {
          const double xc = __shfl_sync(0xffffffffu, v, c) / L11[c][c];
          if (lane == c) v = xc;
          if (lane > c) v = fma(-L11[lane][c], xc, v);
        }
        zp[lane] = (lane < pw) ? v : 0.0;
      }
    }
    __syncthreads();
    if (fail) {
      if (g == 0 && tid == 0) atomicCAS(status, 0, k + 1);
      return;  // all CTAs of the grid take this branch at the same panel
    }
    if (g == 0 && tid == 0) {
      double q = quad_acc;
      for (int c = 0; c < pw; ++c) {
        z[(size_t)k * b + p0 + c] = zp[c];
        q += zp[c] * zp[c];
      }
      quad_acc = q;
    }
    // panel rows below, split across CTAs: X = A21 L11^{-T}; rhs_rows -= X z_p
    const int per = (m + G - 1) / G;
    const int r0 = g * per, r1 = min(m, r0 + per);
    for (int row = r0 + tid; row < r1; row += blockDim.x) {
      double x[kPB];
#pragma unroll
      for (int c = 0; c < kPB; ++c) x[c] = (c < pw) ? A[(size_t)(p0 + c) * b + p0 + pw + row] : 0.0;
      double dz = 0.0;
#pragma unroll
      for (int c = 0; c < kPB; ++c) {
        if (c < pw) {
          double s = x[c];
#pragma unroll
          for (int j = 0; j < c; ++j) s = fma(-x[j], L11[c][j], s);
          x[c] = s / L11[c][c];
          dz = fma(x[c], zp[c], dz);
        }
      }
#pragma unroll
      for (int c = 0; c < kPB; ++c)
        if (c < pw) A[(size_t)(p0 + c) * b + p0 + pw + row] = x[c];
      rk[p0 + pw + row] -= dz;
    }
    __threadfence();
    grid.sync();
    // the factored diagonal block goes back only now: every CTA has finished reading it
    if (g == 0)
      for (int e = tid; e < pw * pw; e += blockDim.x) {
        const int i = e % pw, j = e / pw;
        if (i >= j) A[(size_t)(p0 + j) * b + p0 + i] = L11[i][j];
      }
    // trailing update of the lower triangle in 32 x 32 blocks
    const int mb = (m + 31) / 32;
    const int nblk = mb * (mb + 1) / 2;
    for (int blk = g; blk < nblk; blk += G) {
      int rb = (int)((sqrt(8.0 * blk + 1.0) - 1.0) * 0.5);
      while (rb * (rb + 1) / 2 > blk) --rb;
      while ((rb + 1) * (rb + 2) / 2 <= blk) ++rb;
      const int cb = blk - rb * (rb + 1) / 2;
      const int a0 = rb * 32, c0 = cb * 32;
      __syncthreads();
      for (int t = warp; t < kPB; t += 8) {
        const double* col = A + (size_t)(p0 + t) * b + p0 + pw;
        Pa[lane][t] = (t < pw && a0 + lane < m) ? col[a0 + lane] : 0.0;
        Pc[lane][t] = (t < pw && c0 + lane < m) ? col[c0 + lane] : 0.0;
      }
      __syncthreads();
      const int cl = tid & 31, rl = tid >> 5;  // column cl, rows rl + 8q
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int t = 0; t < pw; ++t) {
        const double pc = Pc[cl][t];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = fma(Pa[rl + 8 * q][t], pc, acc[q]);
      }
      const int cg2 = c0 + cl;
      if (cg2 < m) {
        double* colp = A + (size_t)(p0 + pw + cg2) * b + p0 + pw;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int ag = a0 + rl + 8 * q;
          if (ag < m && ag >= cg2) colp[ag] -= acc[q];
        }
      }
    }
    __threadfence();
    grid.sync();
  }
  if (g == 0 && tid == 0) {
    ldpart[k] = 2.0 * logdet_acc;
    qpart[k] = quad_acc;
  }
}

int launch_potrf(double* D, int n, int b, int k, double* rhs, double* z, double* ldpart, double* qpart,
                 int* status, cudaStream_t s) {
  static int grid_cache = 0;
  if (grid_cache == 0) {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_potrf_coop, 256, 0);
    grid_cache = std::max(1, std::min(64, nsm * std::max(per, 1)));
  }
  int G = grid_cache;
  void* args[] = {&D, &n, &b, &k, &rhs, &z, &ldpart, &qpart, &status};
  cudaLaunchCooperativeKernel((void*)k_potrf_coop, dim3(G), dim3(256), args, 0, s);
  return (int)cudaGetLastError();
}

}  // namespace tlr
