// Cholesky of one diagonal tile per thread-block cluster, then the tile's forward-solve block.
//
// Reference: codes/17_tlr_cholesky_pilot.py:171-177 (scipy.linalg.cholesky of A_kk; a pivot that
// is not positive stops the factorization, failed_at = k) and 230-240 (z_k = L_kk^{-1} rhs_k).
//
// A cluster of kPC CTAs works on the column-major lower triangle of A_kk (L2-resident),
// right-looking in panels of 32 columns, with the cluster's hardware barrier between phases:
//   every CTA factors the 32 x 32 diagonal block redundantly (warp 0, the rows in registers;
//   identical inputs give identical results, so a non-positive pivot stops every CTA at the same
//   panel) and inverts it (lane c forms column c of L11^{-1});
//   the panel rows below are split across the cluster, four threads per row: X = A21 L11^{-T} as
//   independent dot products (no substitution chain), and rhs_rows -= X z_p with
//   z_p = L11^{-1} rhs_p (the fused forward solve);
//   cluster barrier; every CTA stages the whole panel X in shared memory once, and the
//   lower-triangular 32 x 32 blocks of the trailing matrix are split across the cluster
//   (A22 -= X X^T, no block barrier between blocks); cluster barrier.
// Several tiles (one per parameter vector of a batch) are factored by independent clusters of
// one launch.  The status word is read once by rank 0 and shared through distributed shared
// memory, so every CTA of a cluster takes the same branch even when another stream writes the
// status meanwhile.
#include <cooperative_groups.h>

#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace cg = cooperative_groups;

namespace tlr {

constexpr int kPB = 32;  // panel width
constexpr int kPC = 8;   // CTAs per cluster (one cluster per tile)

__global__ void __cluster_dims__(kPC, 1, 1) __launch_bounds__(256)
    k_potrf_cluster(double* TLR_RESTRICT D, int n, int b, int k, double* TLR_RESTRICT rhs, double* TLR_RESTRICT z,
                    double* TLR_RESTRICT ldpart, double* TLR_RESTRICT qpart, int* TLR_RESTRICT status,
                    size_t sD, size_t sV, int sS, int staged) {
  cg::cluster_group cluster = cg::this_cluster();
  const int g = (int)cluster.block_rank(), G = kPC;
  const int bz = blockIdx.x / kPC;  // which tile of the batch
  D += bz * sD;
  rhs += bz * sV;
  z += bz * sV;
  ldpart += bz * (size_t)sS;
  qpart += bz * (size_t)sS;
  status += bz * sS;
  __shared__ double L11[kPB][kPB + 1];
  __shared__ double Li[kPB][kPB + 1];  // L11^{-1}
  __shared__ double dinv[kPB];
  __shared__ double zp[kPB];
  extern __shared__ double Ps[];  // the panel below the diagonal block, b x (kPB + 1), when staged
  __shared__ double Pa[kPB][kPB + 1];
  __shared__ double Pc[kPB][kPB + 1];
  __shared__ int go, fail;
  __shared__ double logdet_acc, quad_acc;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    go = (g == 0) ? (*status == 0) : 0;
    logdet_acc = 0.0;
    quad_acc = 0.0;
  }
  cluster.sync();
  const int ok = *cluster.map_shared_rank(&go, 0);
  cluster.sync();  // rank 0's shared memory stays valid until every CTA has read it
  if (!ok) return;
  const int bk = min(b, n - k * b);
  double* A = D + (size_t)k * b * b;
  double* rk = rhs + (size_t)k * b;
  if (g == 0 && tid == 0) add_work(status, 8, (double)bk * bk * bk / 3.0 + (double)bk * bk, 8.0 * bk * bk);
  for (int p0 = 0; p0 < bk; p0 += kPB) {
    const int pw = min(kPB, bk - p0);
    const int m = bk - p0 - pw;
    if (warp == 0) {
      // Cholesky of the pw x pw diagonal block, lane = row, the row in registers
      double row[kPB];
#pragma unroll
      for (int j = 0; j < kPB; ++j)
        row[j] = (lane < pw && j <= lane) ? A[(size_t)(p0 + j) * b + p0 + lane] : 0.0;
      int bad = 0;
      double dl = 0.0;  // 1 / L11[lane][lane]
#pragma unroll
      for (int c = 0; c < kPB; ++c) {
        if (c < pw && !bad) {
          const double d = __shfl_sync(0xffffffffu, row[c], c);
          if (!(d > 0.0)) {
            bad = 1;  // the same pivot in every lane: the whole warp stops here
          } else {
            // one reciprocal square root per pivot on the column chain (sqrt d = d / sqrt d);
            // an IEEE square root followed by a division costs several times as long here
            const double rsd = rsqrt(d), sd = d * rsd;
            if (lane == c) {
              row[c] = sd;
              dl = rsd;
            }
            if (lane > c) row[c] *= rsd;
#pragma unroll
            for (int j = c + 1; j < kPB; ++j) {
              const double ljc = __shfl_sync(0xffffffffu, row[c], j);
              if (lane >= j) row[j] = fma(-row[c], ljc, row[j]);
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < kPB; ++j) L11[lane][j] = (j <= lane && lane < pw && j < pw) ? row[j] : 0.0;
      if (lane == 0) fail = bad;
      __syncwarp();
      dinv[lane] = (!bad && lane < pw) ? dl : 0.0;
      __syncwarp();
      if (!bad) {
        // column `lane` of L11^{-1} by forward substitution
        double x[kPB];
#pragma unroll
        for (int r = 0; r < kPB; ++r) {
          double s = (r == lane) ? 1.0 : 0.0;
#pragma unroll
          for (int q = 0; q < r; ++q) s = fma(-L11[r][q], x[q], s);
          x[r] = (r < pw) ? s * dinv[r] : 0.0;
        }
#pragma unroll
        for (int r = 0; r < kPB; ++r) Li[r][lane] = x[r];
        __syncwarp();
        // z_p = L11^{-1} rhs_p (one load per lane, broadcast by shuffles), log det
        const double rv = lane < pw ? rk[p0 + lane] : 0.0;
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < kPB; ++q) v = fma(Li[lane][q], __shfl_sync(0xffffffffu, rv, q), v);
        zp[lane] = lane < pw ? v : 0.0;
        if (g == 0) {
          const double ld = warp_sum(lane < pw ? log(L11[lane][lane]) : 0.0);
          if (lane == 0) logdet_acc += ld;
        }
      }
    }
    __syncthreads();
    if (fail) {
      if (g == 0 && tid == 0) atomicCAS(status, 0, k + 1);
      return;  // every CTA of the cluster leaves at the same panel
    }
    // panel rows below, split across the cluster, four threads per row (eight outputs each)
    {
      const int per = (m + G - 1) / G;
      const int r0 = g * per, r1 = min(m, r0 + per);
      const int quarter = tid & 3;
      for (int base = r0; base < r1; base += 64) {  // the same trip count in every thread (shuffles)
        const int row = base + (tid >> 2);
        const bool act = row < r1;
        const size_t ar = (size_t)p0 + pw + (act ? row : 0);
        double a[kPB];
#pragma unroll
        for (int q = 0; q < kPB; ++q) a[q] = (act && q < pw) ? A[(size_t)(p0 + q) * b + ar] : 0.0;
        double xo[8];
        double dz = 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int c = quarter * 8 + u;
          double s = 0.0;
#pragma unroll
          for (int q = 0; q < kPB; ++q) s = fma(a[q], Li[c][q], s);
          xo[u] = s;
          dz = fma(s, zp[c], dz);
        }
        dz += __shfl_xor_sync(0xffffffffu, dz, 1);
        dz += __shfl_xor_sync(0xffffffffu, dz, 2);
        if (act) {
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int c = quarter * 8 + u;
            if (c < pw) A[(size_t)(p0 + c) * b + ar] = xo[u];
          }
          if (quarter == 0) rk[ar] -= dz;
        }
      }
    }
    cluster.sync();
    if (g == 0) {
      for (int e = tid; e < pw * pw; e += blockDim.x) {
        const int i = e % pw, j = e / pw;
        if (i >= j) A[(size_t)(p0 + j) * b + p0 + i] = L11[i][j];
      }
      if (tid == 0) {
        double q = quad_acc;
        for (int c = 0; c < pw; ++c) {
          z[(size_t)k * b + p0 + c] = zp[c];
          q += zp[c] * zp[c];
        }
        quad_acc = q;
      }
    }
    // trailing update of the lower triangle in 32 x 32 blocks.  staged: from the whole panel put in
    // shared memory once (rows below the diagonal block, ld kPB + 1); otherwise (tiles too tall for
    // that) each block's two 32 x 32 panel pieces are loaded from L2 in turn
    if (staged) {
      for (int e = tid; e < m * kPB; e += blockDim.x) {
        const int row = e % m, t = e / m;
        Ps[(size_t)row * (kPB + 1) + t] = t < pw ? A[(size_t)(p0 + t) * b + p0 + pw + row] : 0.0;
      }
      __syncthreads();
    }
    const int mb = (m + 31) / 32;
    const int nblk = mb * (mb + 1) / 2;
    for (int blk = g; blk < nblk; blk += G) {
      if (!staged) {
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
#pragma unroll 8
        for (int t = 0; t < kPB; ++t) {
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
        continue;
      }
      int rb = (int)((sqrt(8.0 * blk + 1.0) - 1.0) * 0.5);
      while (rb * (rb + 1) / 2 > blk) --rb;
      while ((rb + 1) * (rb + 2) / 2 <= blk) ++rb;
      const int cb = blk - rb * (rb + 1) / 2;
      const int a0 = rb * 32, c0 = cb * 32;
      const int cl = tid & 31, rl = tid >> 5;  // column cl, rows rl + 8q
      const int cg2 = c0 + cl;
      double* colp = A + (size_t)(p0 + pw + min(cg2, m - 1)) * b + p0 + pw;
      double old[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {  // the block's current values, loaded before the products
        const int ag = a0 + rl + 8 * q;
        old[q] = (cg2 < m && ag < m && ag >= cg2) ? colp[ag] : 0.0;
      }
      const double* pcr = Ps + (size_t)min(cg2, m - 1) * (kPB + 1);
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int t = 0; t < kPB; ++t) {
        const double pc = pcr[t];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = fma(Ps[(size_t)min(a0 + rl + 8 * q, m - 1) * (kPB + 1) + t], pc, acc[q]);
      }
      if (cg2 < m) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int ag = a0 + rl + 8 * q;
          if (ag < m && ag >= cg2) colp[ag] = old[q] - acc[q];
        }
      }
    }
    cluster.sync();
  }
  if (g == 0 && tid == 0) {
    ldpart[k] = 2.0 * logdet_acc;
    qpart[k] = quad_acc;
  }
}

int launch_potrf(double* D, int n, int b, int k, double* rhs, double* z, double* ldpart, double* qpart,
                 int* status, cudaStream_t s) {
  return launch_potrf_batched(D, n, b, k, rhs, z, ldpart, qpart, status, 1, 0, 0, 0, s);
}

int launch_potrf_batched(double* D, int n, int b, int k, double* rhs, double* z, double* ldpart, double* qpart,
                         int* status, int nbatch, size_t sD, size_t sV, int sS, cudaStream_t s) {
  // the staged panel needs b (kPB + 1) doubles beside the 34 KB of static shared memory
  const size_t sm_staged = (size_t)b * (kPB + 1) * sizeof(double);
  const int staged = sm_staged <= 190 * 1024;
  const size_t sm = staged ? sm_staged : 0;
  cudaFuncSetAttribute(k_potrf_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_potrf_cluster<<<kPC * nbatch, 256, sm, s>>>(D, n, b, k, rhs, z, ldpart, qpart, status, sD, sV, sS, staged);
  return (int)cudaGetLastError();
}

}  // namespace tlr
