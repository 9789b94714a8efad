// Morton (Z-order) permutation of the sites on the device.
//
// Reference: codes/11_tlr_rank_rules.py:40-53.  Coordinates are quantised with a truncating
// cast of c * 2^order (as numpy's astype(int64)), clipped to [0, 2^order - 1]; the x bits go
// to the even and the y bits to the odd positions of the key; the permutation is a STABLE
// argsort of the key.  Here: a counting sort over the 2^(2*order) key values (histogram,
// exclusive scan, scatter), then every bucket holding more than one site is put back into
// ascending input order, which makes the result identical to a stable sort.
#include "tlr_kernels.h"
#include <stdint.h>
#include <climits>

namespace tlr {

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

__global__ void k_morton_keys(const double* xy, int n, int order, unsigned* keys, unsigned* cnt) {
  const int side = 1 << order;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned qx = quantise(xy[2 * i], side), qy = quantise(xy[2 * i + 1], side);
    const unsigned key = spread_bits(qx, order) | (spread_bits(qy, order) << 1);
    keys[i] = key;
    atomicAdd(&cnt[key], 1u);
  }
}

// exclusive scan of nbuckets counts by one CTA of 1024 threads
__global__ void __launch_bounds__(1024) k_scan(const unsigned* cnt, unsigned* off, unsigned* cursor, int nbuckets) {
  __shared__ unsigned part[1024];
  const int per = (nbuckets + 1023) / 1024;
  const int b0 = threadIdx.x * per, b1 = min(nbuckets, b0 + per);
  unsigned s = 0;
  for (int q = b0; q < b1; ++q) s += cnt[q];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int t = 0; t < 1024; ++t) { const unsigned v = part[t]; part[t] = acc; acc += v; }
  }
  __syncthreads();
  unsigned acc = part[threadIdx.x];
  for (int q = b0; q < b1; ++q) { off[q] = acc; cursor[q] = acc; acc += cnt[q]; }
}

__global__ void k_scatter(const unsigned* keys, int n, unsigned* cursor, long long* perm) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned pos = atomicAdd(&cursor[keys[i]], 1u);
    perm[pos] = i;
  }
}

// restore input order inside buckets with more than one site (stable sort semantics)
__global__ void k_fix_ties(const unsigned* cnt, const unsigned* off, int nbuckets, long long* perm) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nbuckets; q += gridDim.x * blockDim.x) {
    const unsigned c = cnt[q];
    if (c < 2) continue;
    long long* p = perm + off[q];
    for (unsigned a = 1; a < c; ++a) {
      const long long v = p[a];
      unsigned b2 = a;
      while (b2 > 0 && p[b2 - 1] > v) { p[b2] = p[b2 - 1]; --b2; }
      p[b2] = v;
    }
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

int launch_morton(const double* xy, int n, int order, unsigned* keys, unsigned* cnt, unsigned* off,
                  unsigned* cursor, long long* perm, cudaStream_t s) {
  const int nbuckets = 1 << (2 * order);
  cudaMemsetAsync(cnt, 0, sizeof(unsigned) * nbuckets, s);
  const int grid = std::max(1, std::min(4096, (n + 255) / 256));
  k_morton_keys<<<grid, 256, 0, s>>>(xy, n, order, keys, cnt);
  k_scan<<<1, 1024, 0, s>>>(cnt, off, cursor, nbuckets);
  k_scatter<<<grid, 256, 0, s>>>(keys, n, cursor, perm);
  k_fix_ties<<<std::min(4096, (nbuckets + 255) / 256), 256, 0, s>>>(cnt, off, nbuckets, perm);
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

}  // namespace tlr
