// The assembled-matrix rule: Sigma^TLR written out densely from the truncated tiles.
//
// Reference: codes/11_tlr_rank_rules.py:74-108 (truncate_tiles: every off-diagonal tile of the
// dense covariance replaced by its rank-r truncation under the rule, in place, symmetric) and
// 11:121-126 (make_cov), used with a dense Cholesky by 11:112-120 and 11:130-138; the same
// matrix is what codes/19_tlr_mcmc_gpu.py:51-123 (Likelihood.truncate) builds on the GPU.
//
// Here the truncations are those of the plan's initial compression (sketch + exact residual,
// the reference's ranks), so only the write-out is new: one CTA per 32 x 32 block of a tile
// (i, j), i >= j.  A diagonal block is Sigma_ii itself (Matern + nugget); an off-diagonal block
// is (U_ij V_ij^T) restricted to the block, staged in shared memory and stored twice, at (i, j)
// and transposed at (j, i), both with coalesced columns.  K is symmetric, so its storage order
// (row- or column-major, leading dimension ldk) does not matter.
#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace tlr {

__global__ void __launch_bounds__(256) k_assemble(const double* TLR_RESTRICT xy, int n, int b, double sigma2,
                                                 double inv_range, int nu5, double nugget,
                                                 const double* TLR_RESTRICT U, const double* TLR_RESTRICT V,
                                                 const int* TLR_RESTRICT rank, int cap, double* TLR_RESTRICT K,
                                                 long long ldk, const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  // blockIdx.z -> tile (i, j), i >= j, in the order (0,0), (1,0), (1,1), (2,0), ...
  int z = blockIdx.z, i = 0;
  while (z > i) { z -= i + 1; ++i; }
  const int j = z;
  const int bi = min(b, n - i * b), bj = min(b, n - j * b);
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  if (r0 >= bi || c0 >= bj) return;
  __shared__ double blk[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  const double2* p2 = reinterpret_cast<const double2*>(xy);
  if (i == j) {
    const int c = c0 + tx;
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + ty + 8 * q;
      if (r < bi && c < bj) {
        const double2 pa = p2[i * b + r], pc = p2[j * b + c];
        const double v = matern_cov(pa.x, pa.y, pc.x, pc.y, sigma2, inv_range, nu5) + (r == c ? nugget : 0.0);
        K[(long long)(j * b + c) * ldk + i * b + r] = v;
      }
    }
    return;
  }
  const int t = i * (i - 1) / 2 + j;
  const int rk = rank[t];
  const double* Ut = U + (size_t)t * b * cap;
  const double* Vt = V + (size_t)t * b * cap;
  // blk[row][col] = sum_q U[r0 + row, q] V[c0 + col, q]; thread (tx, ty) owns column tx, rows ty + 8q
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const int c = c0 + tx;
  for (int q = 0; q < rk; ++q) {
    const double vc = c < bj ? Vt[(size_t)q * b + c] : 0.0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = r0 + ty + 8 * u;
      acc[u] = fma(r < bi ? Ut[(size_t)q * b + r] : 0.0, vc, acc[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) blk[ty + 8 * u][tx] = acc[u];
  __syncthreads();
  // (i, j): column c0 + tx of tile j, rows r0 .. r0 + 31 of tile i (lanes run down a column)
  for (int u = 0; u < 4; ++u) {
    const int col = ty + 8 * u;  // column within the block
    const int r = r0 + tx;
    if (c0 + col < bj && r < bi) K[(long long)(j * b + c0 + col) * ldk + i * b + r] = blk[tx][col];
  }
  // (j, i): the transpose, column r0 + row of tile i, rows c0 .. c0 + 31 of tile j
  for (int u = 0; u < 4; ++u) {
    const int row = ty + 8 * u;
    const int cc = c0 + tx;
    if (r0 + row < bi && cc < bj) K[(long long)(i * b + r0 + row) * ldk + j * b + cc] = blk[row][tx];
  }
}

int launch_assemble(const double* xy, int n, int b, double sigma2, double inv_range, int nu5, double nugget,
                    const double* U, const double* V, const int* rank, int cap, double* K, long long ldk,
                    const int* status, cudaStream_t s) {
  const int nB = (n + b - 1) / b;
  const long long tiles = (long long)nB * (nB + 1) / 2;
  if (tiles > 65535) return (int)cudaErrorInvalidConfiguration;
  const int nsub = (b + 31) / 32;
  dim3 grid((unsigned)nsub, (unsigned)nsub, (unsigned)tiles);
  k_assemble<<<grid, 256, 0, s>>>(xy, n, b, sigma2, inv_range, nu5, nugget, U, V, rank, cap, K, ldk, status);
  return (int)cudaGetLastError();
}

}  // namespace tlr
