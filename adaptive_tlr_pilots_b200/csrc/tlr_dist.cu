// Exchange buffers of the block-row cyclic factorization (codes/13_multigpu_tile_cholesky.py:45-79:
// block row i lives on rank i % world; at step k the owner of row k factors the diagonal tile,
// every rank receives it, solves its own panel tiles (i, k) and receives everyone's, then updates
// its own trailing rows).  The kernels here only pack and unpack plain device buffers; the host
// moves them between ranks (NCCL through torch.distributed, or device copies between plans that
// share one GPU).
//
// Diagonal buffer (8 + b b + b doubles): [status, 7 unused | L_kk (b x b, column-major, ld b) | z_k].
// Panel buffer of one rank at step k (tlr_dist_panel_doubles): [status, 7 unused | slot 0 | slot 1
// ...], one slot per row i > k the rank owns, ascending, each [r, i, 6 unused | U (b x cap) | V
// (b x cap)] with the first r columns of U and V filled.
// Sums buffer (2 nB + ntiles + world): [log det parts | quadratic parts | initial ranks of the
// rank's own tiles, zero elsewhere | status at the rank's own position, zero elsewhere], summed
// over the ranks.
#include "tlr_kernels.h"

namespace tlr {

namespace {

__device__ __forceinline__ int dist_tidx(int i, int j) { return i * (i - 1) / 2 + j; }

// first row after k that rank `src` owns, and how many it owns below row k
__host__ __device__ inline int dist_first_row(int k, int src, int world) {
  return k + 1 + (((src - (k + 1)) % world) + world) % world;
}
__host__ __device__ inline int dist_rows_after(int k, int nB, int src, int world) {
  const int f = dist_first_row(k, src, world);
  return f < nB ? (nB - 1 - f) / world + 1 : 0;
}

__global__ void k_dist_pack_diag(const double* D, const double* z, const int* status, int n, int b, int k,
                                 double* buf) {
  const int bk = min(b, n - k * b);
  const double* Dk = D + (size_t)k * b * b;
  const size_t total = (size_t)b * b + b;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    double v;
    if (e < (size_t)b * b) v = Dk[e];
    else v = (int)(e - (size_t)b * b) < bk ? z[(size_t)k * b + (e - (size_t)b * b)] : 0.0;
    buf[8 + e] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x < 8) buf[threadIdx.x] = threadIdx.x == 0 ? (double)*status : 0.0;
}

__global__ void k_dist_unpack_diag(double* D, double* z, int* status, int n, int b, int k, const double* buf) {
  const int bk = min(b, n - k * b);
  double* Dk = D + (size_t)k * b * b;
  const size_t total = (size_t)b * b + bk;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    if (e < (size_t)b * b) Dk[e] = buf[8 + e];
    else z[(size_t)k * b + (e - (size_t)b * b)] = buf[8 + e];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && *status == 0) *status = (int)buf[0];
}

// one CTA per (slot, U or V)
__global__ void k_dist_pack_panel(const double* U, const double* V, const int* rank, const int* status, int n, int b,
                                  int k, int nB, int cap, int prank, int pworld, double* buf) {
  const int q = blockIdx.x, side = blockIdx.y;
  const size_t stride = 8 + 2 * (size_t)b * cap;
  if (q == 0 && side == 0 && threadIdx.x < 8) buf[threadIdx.x] = threadIdx.x == 0 ? (double)*status : 0.0;
  if (q >= dist_rows_after(k, nB, prank, pworld)) return;
  const int i = dist_first_row(k, prank, pworld) + q * pworld;
  const int t = dist_tidx(i, k);
  const int r = min(rank[t], cap);
  double* slot = buf + 8 + (size_t)q * stride;
  if (side == 0 && threadIdx.x < 8) slot[threadIdx.x] = threadIdx.x == 0 ? (double)r : threadIdx.x == 1 ? (double)i : 0.0;
  const double* src = (side == 0 ? U : V) + (size_t)t * b * cap;
  double* dst = slot + 8 + (size_t)side * b * cap;
  const size_t m = (size_t)b * r;
  for (size_t e = threadIdx.x; e < m; e += blockDim.x) dst[e] = src[e];
}

// one CTA per (slot, source rank, U or V); every rank but this one
__global__ void k_dist_unpack_panel(double* U, double* V, int* rank, int* status, int n, int b, int k, int nB,
                                    int cap, int prank, int pworld, const double* gathered, size_t len) {
  const int q = blockIdx.x, src = blockIdx.y >> 1, side = blockIdx.y & 1;
  if (q == 0 && blockIdx.y == 0 && threadIdx.x == 0 && *status == 0)
    for (int w = 0; w < pworld; ++w) {  // the first failure in rank order
      const int st = w == prank ? 0 : (int)gathered[(size_t)w * len];
      if (st != 0) { *status = st; break; }
    }
  if (src == prank || q >= dist_rows_after(k, nB, src, pworld)) return;
  const size_t stride = 8 + 2 * (size_t)b * cap;
  const double* slot = gathered + (size_t)src * len + 8 + (size_t)q * stride;
  const int i = dist_first_row(k, src, pworld) + q * pworld;
  const int t = dist_tidx(i, k);
  const int r = min((int)slot[0], cap);
  if (side == 0 && threadIdx.x == 0) rank[t] = r;
  double* dst = (side == 0 ? U : V) + (size_t)t * b * cap;
  const double* from = slot + 8 + (size_t)side * b * cap;
  const size_t m = (size_t)b * r;
  for (size_t e = threadIdx.x; e < m; e += blockDim.x) dst[e] = from[e];
}

__global__ void k_dist_pack_sums(const double* ldpart, const double* qpart, const int* rank0, const int* ti,
                                 const int* status, int nB, int ntiles, int prank, int pworld, double* buf) {
  const int total = 2 * nB + ntiles + pworld;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    double v = 0.0;
    if (e < nB) v = e % pworld == prank ? ldpart[e] : 0.0;
    else if (e < 2 * nB) v = (e - nB) % pworld == prank ? qpart[e - nB] : 0.0;
    else if (e < 2 * nB + ntiles) v = ti[e - 2 * nB] % pworld == prank ? (double)rank0[e - 2 * nB] : 0.0;
    else v = e - 2 * nB - ntiles == prank ? (double)*status : 0.0;
    buf[e] = v;
  }
}

__global__ void k_dist_unpack_sums(double* ldpart, double* qpart, int* rank0, int* status, int nB, int ntiles,
                                   int pworld, const double* sums) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * nB + ntiles; e += gridDim.x * blockDim.x) {
    if (e < nB) ldpart[e] = sums[e];
    else if (e < 2 * nB) qpart[e - nB] = sums[e];
    else rank0[e - 2 * nB] = (int)sums[e];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // every rank settles on the first failure in rank order
    int st = 0;
    for (int w = 0; w < pworld && st == 0; ++w) st = (int)sums[2 * nB + ntiles + w];
    *status = st;
  }
}

}  // namespace

size_t dist_panel_doubles(int b, int cap, int k, int nB, int pworld) {
  int most = 0;
  if (k < 0) {
    most = (nB - 1 + pworld - 1) / pworld;  // step 0 holds the most rows
  } else {
    for (int w = 0; w < pworld; ++w) most = std::max(most, dist_rows_after(k, nB, w, pworld));
  }
  return 8 + (size_t)most * (8 + 2 * (size_t)b * cap);
}

int launch_dist_pack_diag(const double* D, const double* z, const int* status, int n, int b, int k, double* buf,
                          cudaStream_t s) {
  k_dist_pack_diag<<<std::max(1, std::min(256, (b * b + 255) / 256)), 256, 0, s>>>(D, z, status, n, b, k, buf);
  return (int)cudaGetLastError();
}

int launch_dist_unpack_diag(double* D, double* z, int* status, int n, int b, int k, const double* buf,
                            cudaStream_t s) {
  k_dist_unpack_diag<<<std::max(1, std::min(256, (b * b + 255) / 256)), 256, 0, s>>>(D, z, status, n, b, k, buf);
  return (int)cudaGetLastError();
}

int launch_dist_pack_panel(const double* U, const double* V, const int* rank, const int* status, int n, int b, int k,
                           int nB, int cap, int prank, int pworld, double* buf, cudaStream_t s) {
  const int slots = std::max(1, dist_rows_after(k, nB, prank, pworld));
  k_dist_pack_panel<<<dim3(slots, 2), 256, 0, s>>>(U, V, rank, status, n, b, k, nB, cap, prank, pworld, buf);
  return (int)cudaGetLastError();
}

int launch_dist_unpack_panel(double* U, double* V, int* rank, int* status, int n, int b, int k, int nB, int cap,
                             int prank, int pworld, const double* gathered, size_t len, cudaStream_t s) {
  int slots = 1;
  for (int w = 0; w < pworld; ++w) slots = std::max(slots, dist_rows_after(k, nB, w, pworld));
  k_dist_unpack_panel<<<dim3(slots, 2 * pworld), 256, 0, s>>>(U, V, rank, status, n, b, k, nB, cap, prank, pworld,
                                                              gathered, len);
  return (int)cudaGetLastError();
}

int launch_dist_pack_sums(const double* ldpart, const double* qpart, const int* rank0, const int* ti,
                          const int* status, int nB, int ntiles, int prank, int pworld, double* buf, cudaStream_t s) {
  const int total = 2 * nB + ntiles + pworld;
  k_dist_pack_sums<<<std::min(1024, (total + 255) / 256), 256, 0, s>>>(ldpart, qpart, rank0, ti, status, nB, ntiles,
                                                                       prank, pworld, buf);
  return (int)cudaGetLastError();
}

int launch_dist_unpack_sums(double* ldpart, double* qpart, int* rank0, int* status, int nB, int ntiles, int pworld,
                            const double* sums, cudaStream_t s) {
  const int total = 2 * nB + ntiles;
  k_dist_unpack_sums<<<std::max(1, std::min(1024, (total + 255) / 256)), 256, 0, s>>>(ldpart, qpart, rank0, status,
                                                                                       nB, ntiles, pworld, sums);
  return (int)cudaGetLastError();
}

}  // namespace tlr
