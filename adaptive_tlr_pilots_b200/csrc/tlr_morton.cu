// Morton (Z-order) permutation of the sites on the device.
//
// Reference: codes/11_tlr_rank_rules.py:40-53.  Coordinates are quantised with a truncating
// cast of c * 2^order (as numpy's astype(int64)), clipped to [0, 2^order - 1]; the x bits go
// to the even and the y bits to the odd positions of the key; the permutation is a STABLE
// argsort of the key (equal keys keep their input order).
//
// Here: a least-significant-digit radix sort of (key, index) pairs.  Each pass orders by one
// digit of the key and is stable, so after the last pass equal keys are still in input order:
// the stable argsort by construction, with the same amount of work whatever the key
// distribution (many sites clipped into one cell, NaN coordinates, exact duplicates).
//   * up to 8 key bits: one pass of up to 8 bits; otherwise three passes of ceil(bits / 3)
//     bits (order <= 12, so at most 8 bits, 256 digit values).  The odd pass count lets the
//     passes ping-pong between the work array and the caller's perm buffer (n int64 = room for
//     n keys + n indices) and end with the last pass writing perm itself;
//   * a pass: per tile of 2,048 consecutive pairs a digit histogram, an exclusive scan of the
//     (digit, tile) counts in digit-major order, then a scatter in which each pair goes to
//     scan[digit][tile] + (pairs of the same digit earlier in the tile).  Inside a tile the
//     pairs are taken 256 at a time in input order; a pair's rank among its warp's lanes of the
//     same digit comes from __match_any_sync, the earlier warps' counts from shared memory.
#include "tlr_kernels.h"
#include <stdint.h>
#include <climits>

namespace tlr {

namespace {
constexpr int kMtThreads = 256;
constexpr int kMtPer = 8;                       // pairs per thread per tile
constexpr int kMtTile = kMtThreads * kMtPer;    // 2,048 pairs per tile

int digit_bits(int order) {
  const int bits = 2 * order;
  return bits <= 8 ? bits : (bits + 2) / 3;
}
int digit_passes(int order) { return 2 * order <= 8 ? 1 : 3; }
}  // namespace

size_t morton_work_words(int n, int order) {
  const size_t ntiles = ((size_t)n + kMtTile - 1) / kMtTile;
  return 2 * (size_t)n + ((size_t)1 << digit_bits(order)) * ntiles;
}

__device__ __forceinline__ unsigned quantise(double v, int side) {
  // numpy: (v * side).astype(int64) truncates; NaN and out-of-range values become INT64_MIN.
  const double s = v * (double)side;
  long long q;
  if (!(fabs(s) < 9.0e18)) q = LLONG_MIN;
  else q = (long long)s;
  if (q < 0) q = 0;
  if (q > side - 1) q = side - 1;
  return (unsigned)q;
}

__device__ __forceinline__ unsigned spread_bits(unsigned v, int order) {
  unsigned out = 0;
  for (int bit = 0; bit < order; ++bit) out |= ((v >> bit) & 1u) << (2 * bit);
  return out;
}

__global__ void k_morton_keys(const double* xy, int n, int order, unsigned* keys, unsigned* idx) {
  const int side = 1 << order;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned qx = quantise(xy[2 * i], side), qy = quantise(xy[2 * i + 1], side);
    keys[i] = spread_bits(qx, order) | (spread_bits(qy, order) << 1);
    idx[i] = (unsigned)i;
  }
}

// hist[d * ntiles + tile] = number of pairs of the tile whose digit (key >> shift) & mask is d
__global__ void __launch_bounds__(kMtThreads) k_digit_hist(const unsigned* keys, int n, int shift, unsigned mask,
                                                           unsigned* hist, int ntiles) {
  __shared__ unsigned cnt[256];
  const int tile = blockIdx.x, tid = threadIdx.x;
  cnt[tid] = 0;
  __syncthreads();
  for (int r = 0; r < kMtPer; ++r) {
    const long i = (long)tile * kMtTile + r * kMtThreads + tid;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & mask], 1u);
  }
  __syncthreads();
  if ((unsigned)tid <= mask) hist[(size_t)tid * ntiles + tile] = cnt[tid];
}

// exclusive scan of `total` counts in place, one CTA of 1,024 threads (contiguous chunks)
__global__ void __launch_bounds__(1024) k_scan_counts(unsigned* c, long total) {
  __shared__ unsigned part[1024];
  const long per = (total + 1023) / 1024;
  const long b0 = threadIdx.x * per, b1 = min(total, b0 + per);
  unsigned s = 0;
  for (long q = b0; q < b1; ++q) s += c[q];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int t = 0; t < 1024; ++t) { const unsigned v = part[t]; part[t] = acc; acc += v; }
  }
  __syncthreads();
  unsigned acc = part[threadIdx.x];
  for (long q = b0; q < b1; ++q) { const unsigned v = c[q]; c[q] = acc; acc += v; }
}

// Stable scatter of one pass.  With perm_out set (last pass) only the indices are written, as int64.
__global__ void __launch_bounds__(kMtThreads) k_digit_scatter(const unsigned* keys_in, const unsigned* idx_in, int n,
                                                              int shift, unsigned mask, const unsigned* scan,
                                                              int ntiles, unsigned* keys_out, unsigned* idx_out,
                                                              long long* perm_out) {
  __shared__ unsigned run[256];                        // pairs of each digit placed by earlier rounds
  __shared__ unsigned wc[kMtThreads / 32][256];        // this pass: pairs of each digit per warp
  const int tile = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  run[tid] = 0;
  for (int r = 0; r < kMtPer; ++r) {
#pragma unroll
    for (int w = 0; w < kMtThreads / 32; ++w) wc[w][tid] = 0;
    __syncthreads();
    const long i = (long)tile * kMtTile + r * kMtThreads + tid;
    const bool valid = i < n;
    unsigned key = 0, id = 0, d = 0x100u;  // 0x100: no pair (past the end); never a digit
    if (valid) {
      key = keys_in[i];
      id = idx_in[i];
      d = (key >> shift) & mask;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned rank = __popc(peers & lt);
    if (valid && lane == __ffs(peers) - 1) wc[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      unsigned pre = 0;
      for (int w = 0; w < warp; ++w) pre += wc[w][d];
      const size_t pos = (size_t)scan[(size_t)d * ntiles + tile] + run[d] + pre + rank;
      if (perm_out) perm_out[pos] = (long long)id;
      else { keys_out[pos] = key; idx_out[pos] = id; }
    }
    __syncthreads();
    unsigned add = 0;
#pragma unroll
    for (int w = 0; w < kMtThreads / 32; ++w) add += wc[w][tid];
    run[tid] += add;
    __syncthreads();
  }
}

__global__ void k_gather(const double* xy_in, const double* y_in, const long long* perm, int n, double* xy_out,
                         double* y_out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const long long p = perm[i];
    xy_out[2 * i] = xy_in[2 * p];
    xy_out[2 * i + 1] = xy_in[2 * p + 1];
    if (y_in) y_out[i] = y_in[p];
  }
}

int launch_morton(const double* xy, int n, int order, unsigned* work, long long* perm, cudaStream_t s) {
  const int w = digit_bits(order), passes = digit_passes(order);
  const unsigned mask = (1u << w) - 1u;
  const int ntiles = (int)(((long)n + kMtTile - 1) / kMtTile);
  unsigned* keysA = work;
  unsigned* idxA = work + n;
  unsigned* hist = work + 2 * (size_t)n;
  unsigned* keysB = reinterpret_cast<unsigned*>(perm);  // the caller's n int64 = n keys + n indices
  unsigned* idxB = keysB + n;
  const long nh = (long)(mask + 1) * ntiles;
  cudaGetLastError();  // an earlier launch's error must not be reported as this call's
  const int grid = std::max(1, std::min(4096, (n + 255) / 256));
  k_morton_keys<<<grid, 256, 0, s>>>(xy, n, order, keysA, idxA);
  for (int p = 0; p < passes; ++p) {
    const bool from_a = (p % 2) == 0, last = p == passes - 1;
    const unsigned* kin = from_a ? keysA : keysB;
    const unsigned* iin = from_a ? idxA : idxB;
    k_digit_hist<<<ntiles, kMtThreads, 0, s>>>(kin, n, p * w, mask, hist, ntiles);
    k_scan_counts<<<1, 1024, 0, s>>>(hist, nh);
    k_digit_scatter<<<ntiles, kMtThreads, 0, s>>>(kin, iin, n, p * w, mask, hist, ntiles,
                                                  from_a ? keysB : keysA, from_a ? idxB : idxA,
                                                  last ? perm : nullptr);
  }
  return (int)cudaGetLastError();
}

int launch_gather_sites(const double* xy_in, const double* y_in, const long long* perm, int n, double* xy_out,
                        double* y_out, cudaStream_t s) {
  const int grid = std::max(1, std::min(4096, (n + 255) / 256));
  k_gather<<<grid, 256, 0, s>>>(xy_in, y_in, perm, n, xy_out, y_out);
  return (int)cudaGetLastError();
}

__global__ void k_fill_int(int* p, int v, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) p[i] = v;
}

int launch_fill_int(int* p, int v, int count, cudaStream_t s) {
  if (count <= 0) return 0;
  k_fill_int<<<std::min(1024, (count + 255) / 256), 256, 0, s>>>(p, v, count);
  return (int)cudaGetLastError();
}

__global__ void k_set_params(int* control, EvalParams prm) {
  for (int i = threadIdx.x; i < (int)kControlInts; i += blockDim.x) control[i] = 0;
  if (threadIdx.x == 0) *reinterpret_cast<EvalParams*>(control + kControlInts) = prm;
}

int launch_set_params(int* control, EvalParams prm, cudaStream_t s) {
  k_set_params<<<1, 128, 0, s>>>(control, prm);
  return (int)cudaGetLastError();
}

}  // namespace tlr
