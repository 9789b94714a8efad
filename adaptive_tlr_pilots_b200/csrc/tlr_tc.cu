// Tensor-core (tcgen05) GEMM for the mixed-precision path: C = alpha op(A) op(B) + beta C with FP64
// operands and result, products formed on the 5th-generation tensor cores as split TF32
// ("3xTF32": x = hi + lo with hi, lo TF32, A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi) accumulated in
// FP32 in tensor memory.  Relative accuracy is that of FP32 (about 1e-7 per product), which keeps
// the selected-inversion gradient within ~1e-5 of the FP64 one (single-pass TF32 loses ~1e-2 on
// the range component).
//
// One CTA of 512 threads computes a 128 x N_TILE output tile (N_TILE = 128): the accumulator is
// 128 TMEM lanes x 128 columns.  K advances in slices of 16 through a ring of six shared-memory
// stages.  Each stage first receives the raw FP64 slice of A and of B by cp.async (16-byte copies
// when every row start is 16-byte aligned, else 8-byte; rows and k beyond the matrix arrive as
// zeros), five slices ahead of the one being converted, so the copies' latency hides behind the
// conversion and the MMAs of the slices before.  The threads then read their four k values of
// one tile row (thread = row + 128 x k-group), and, after a block barrier, overwrite the same
// stage with the split TF32 values in the canonical K-major, no-swizzle UMMA layout (core
// matrices of 8 rows x 16 bytes; rows of a core matrix 16 B apart, 8-row groups 128 B apart, the
// two 16-byte K halves of one MMA 2048 B apart): a double and its (hi, lo) pair take the same 8
// bytes, so the conversion fits in place.  After a fence for the async proxy and a barrier,
// thread 0 issues 2 K-steps x 3 tcgen05.mma.kind::tf32 and commits them to the stage's mbarrier;
// the stage is refilled once that commit completes.  The MMA sequence (K-steps of 8 in order,
// three products each) is the same for any slice length, so results do not depend on it.
// Waits on the mbarriers are bounded: on timeout the kernel sets an error status, lets its copies
// land, frees its tensor memory and returns.
#include <stdint.h>

#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace tlr {

constexpr int kTcM = 128;
constexpr int kTcN = 128;
constexpr int kTcBK = 16;                          // k per slice: two MMA K-steps
constexpr int kTcStages = 6;
constexpr int kTcThreads = 512;                    // thread = tile row (0..127) + 128 x k-group (0..3)
constexpr int kTcRawKS = kTcBK + 2;                // row stride (doubles) of a k-contiguous raw slice
constexpr int kTcOpBytes = kTcM * kTcRawKS * 8;    // one operand's region: 18,432 B >= 16 KB of hi + lo
constexpr int kTcStageBytes = 2 * kTcOpBytes;      // A region, then B region
static_assert(kTcM == kTcN && kTcThreads == 4 * kTcM && kTcBK == 16, "thread map assumes 128 x 128 x 16");
static_assert(kTcStageBytes * kTcStages + 1024 <= 227 * 1024, "stages exceed shared memory");
constexpr long long kTcWaitLimit = 1ll << 23;  // polls of about 140 ns on B200: about 1.2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// K-major, no-swizzle shared-memory matrix descriptor (SM100 UMMA): start address, leading
// byte offset (between the two 16-byte K halves), stride byte offset (between 8-row groups), all
// in 16-byte units; version 1; layout type 0 (no swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;
}

// instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N = kTcN
__device__ __forceinline__ uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; false on timeout
__device__ __forceinline__ bool mbar_wait_n(uint32_t mbar, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; ++it)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  return mbar_wait_n(mbar, parity, kTcWaitLimit);
}

// Self-test of the timeout path: the GEMM's set-up (tensor memory allocated, an mbarrier
// initialised), then a bounded wait on a phase that nothing completes; when the wait runs out
// the kernel frees its tensor memory and reports TLR_ERR_TIMEOUT (-7), as k_gemm_tc3 does.
__global__ void k_wait_selftest(long long limit, int* status) {
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_sh;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(32));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  bool ok = true;
  if (tid == 0) ok = mbar_wait_n(smem_u32(&mbar), 0u, limit);  // no arrival: runs out
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base_sh), "r"(32));
  if (tid == 0) *status = ok ? 0 : -7;
}

// One operand's raw FP64 slice global -> shared by cp.async: 128 tile rows x 16 k from row0 and
// k0, zeros beyond `rows` and K.  kcont: k is the contiguous index in global memory (element
// (row, k) at X[row * ld + k]); the slice is then stored [row][kTcRawKS], else [k][128] (element
// at X[k * ld + row]).  VEC doubles per copy (2: X and ld keep every copy 16-byte aligned).
template <int VEC>
__device__ __forceinline__ void tc_load_slice(double* raw, const double* X, int ld, int rows, int row0, int K, int k0,
                                              int kcont, int tid) {
  constexpr int kChunks = kTcM * kTcBK / VEC;
#pragma unroll
  for (int i = 0; i < kChunks / kTcThreads; ++i) {
    const int q = tid + i * kTcThreads;
    int row, k, nv;
    const double* src;
    double* dst;
    if (kcont) {
      row = q / (kTcBK / VEC);
      k = (q % (kTcBK / VEC)) * VEC;
      nv = row0 + row < rows ? min(VEC, K - (k0 + k)) : 0;
      src = X + (size_t)(row0 + row) * ld + (k0 + k);
      dst = raw + row * kTcRawKS + k;
    } else {
      k = q / (kTcM / VEC);
      row = (q % (kTcM / VEC)) * VEC;
      nv = k0 + k < K ? min(VEC, rows - (row0 + row)) : 0;
      src = X + (size_t)(k0 + k) * ld + (row0 + row);
      dst = raw + k * kTcM + row;
    }
    if (nv <= 0) {  // nothing to read: zeros, from a valid address
      nv = 0;
      src = X;
    }
    if (VEC == 2) cp_async16(dst, src, nv * 8);
    else cp_async8(dst, src, nv * 8);
  }
}

// k values 4g .. 4g + 3 of tile row r from a raw slice
__device__ __forceinline__ void tc_read4(const double* raw, int kcont, int r, int g, double (&x)[4]) {
  if (kcont) {
    const double2 u = *reinterpret_cast<const double2*>(raw + r * kTcRawKS + 4 * g);
    const double2 v = *reinterpret_cast<const double2*>(raw + r * kTcRawKS + 4 * g + 2);
    x[0] = u.x;
    x[1] = u.y;
    x[2] = v.x;
    x[3] = v.y;
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = raw[(4 * g + c) * kTcM + r];
  }
}

// split x = hi + lo (both TF32) and store them in the UMMA layout: hi at `out`, lo 8 KB after
__device__ __forceinline__ void tc_write4(float* out, const double (&x)[4], int r, int g) {
  float4 h, l;
  float* ph = &h.x;
  float* pl = &l.x;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float f = (float)x[c];
    const float fh = __uint_as_float(to_tf32(f));
    ph[c] = fh;
    pl[c] = __uint_as_float(to_tf32(f - fh));
  }
  *reinterpret_cast<float4*>(out + g * (kTcM * 4) + r * 4) = h;
  *reinterpret_cast<float4*>(out + kTcM * kTcBK + g * (kTcM * 4) + r * 4) = l;
}

template <int VEC>
__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_tc3(const GemmJob* TLR_RESTRICT jobs, int* TLR_RESTRICT status,
                                                 int kind) {
  if (*status != 0) return;
  const GemmJob jb = jobs[blockIdx.z];
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
  if (m0 >= jb.M || n0 >= jb.N) return;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t mbar[kTcStages];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int timed_out;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(kTcN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])));
    asm volatile("fence.mbarrier_init.release.cluster;");
    timed_out = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem_d = tmem_base_sh;
  const uint32_t idesc = umma_idesc_tf32(kTcM, kTcN);
  const int nk = (jb.K + kTcBK - 1) / kTcBK;
  const int kcA = jb.transA ? 1 : 0, kcB = jb.transB ? 0 : 1;
  const int trow = tid & (kTcM - 1), kg = tid >> 7;
  // copies of slice s into its stage, committed as one group (an empty group past the end keeps
  // the count of groups per slice uniform)
  auto issue = [&](int s) {
    if (s < nk) {
      double* raw = reinterpret_cast<double*>(tc_smem + (s % kTcStages) * kTcStageBytes);
      tc_load_slice<VEC>(raw, jb.A, jb.lda, jb.M, m0, jb.K, s * kTcBK, kcA, tid);
      tc_load_slice<VEC>(raw + kTcOpBytes / 8, jb.B, jb.ldb, jb.N, n0, jb.K, s * kTcBK, kcB, tid);
    }
    cp_async_commit();
  };
#pragma unroll 1
  for (int s = 0; s < kTcStages - 1; ++s) issue(s);
  cp_async_wait<kTcStages - 2>();  // slice 0 landed
  __syncthreads();
  int fail = 0, bad = 0;
#pragma unroll 1
  for (int s = 0; s < nk; ++s) {
    const int st = s % kTcStages;
    unsigned char* base = tc_smem + st * kTcStageBytes;
    double xa[4], xb[4];
    tc_read4(reinterpret_cast<const double*>(base), kcA, trow, kg, xa);
    tc_read4(reinterpret_cast<const double*>(base + kTcOpBytes), kcB, trow, kg, xb);
    if (__syncthreads_or(bad)) {  // every raw read of the stage is done (or a wait ran out)
      fail = 1;
      break;
    }
    tc_write4(reinterpret_cast<float*>(base), xa, trow, kg);
    tc_write4(reinterpret_cast<float*>(base + kTcOpBytes), xb, trow, kg);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    cp_async_wait<kTcStages - 3>();  // slice s + 1 landed; the barrier publishes it with this stage
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t aH = smem_u32(base), aL = aH + kTcM * kTcBK * 4;
      const uint32_t bH = smem_u32(base + kTcOpBytes), bL = bH + kTcN * kTcBK * 4;
      const uint32_t lboA = kTcM * 16, lboB = kTcN * 16, sbo = 128;
#pragma unroll
      for (int ks = 0; ks < kTcBK / 8; ++ks) {
        const uint32_t oa = ks * 2 * kTcM * 16, ob = ks * 2 * kTcN * 16;
        const uint64_t dAh = umma_desc(aH + oa, lboA, sbo), dAl = umma_desc(aL + oa, lboA, sbo);
        const uint64_t dBh = umma_desc(bH + ob, lboB, sbo), dBl = umma_desc(bL + ob, lboB, sbo);
        const uint32_t first = (s == 0 && ks == 0) ? 0u : 1u;
        mma_tf32(tmem_d, dAh, dBh, idesc, first);
        mma_tf32(tmem_d, dAh, dBl, idesc, 1u);
        mma_tf32(tmem_d, dAl, dBh, idesc, 1u);
      }
      mma_commit(smem_u32(&mbar[st]));
    }
    // slice s + 5 refills the stage of slice s - 1 once the MMAs that read it are done
    const int nxt = s + kTcStages - 1;
    if (s >= 1 && nxt < nk && !bad) {
      const int prev = s - 1;
      if (!mbar_wait(smem_u32(&mbar[prev % kTcStages]), (uint32_t)((prev / kTcStages) & 1))) bad = 1;
    }
    if (!bad) issue(nxt);
    else cp_async_commit();
  }
  cp_async_wait<0>();  // no copy in flight when the kernel leaves
  if (__syncthreads_or(bad | fail)) fail = 1;
  // wait for the last commit (it covers every MMA issued before it)
  if (!fail && nk > 0 && tid == 0) {
    const int last = nk - 1;
    if (!mbar_wait(smem_u32(&mbar[last % kTcStages]), (uint32_t)((last / kTcStages) & 1))) timed_out = 1;
  }
  if (fail && tid == 0) timed_out = 1;
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const bool ok = !timed_out;
  if (ok) {
    // warp w reads TMEM lane quarter w % 4 (the lanes a warp may access) and column quarter w / 4
    const int quarter = warp & 3, part = warp >> 2, nparts = kTcThreads / 128;
    const int row = quarter * 32 + lane;
    const int gm = m0 + row;
    for (int c0 = part * (kTcN / nparts); c0 < (part + 1) * (kTcN / nparts); c0 += 8) {
      uint32_t r[8];
      const uint32_t taddr = tmem_d + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                   : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (nk == 0)
#pragma unroll
        for (int q = 0; q < 8; ++q) r[q] = 0u;
      if (gm < jb.M) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int gn = n0 + c0 + q;
          if (gn >= jb.N) break;
          double* cc = jb.ccol ? jb.ccol[gn] : jb.C + (size_t)gn * jb.ldc;
          const double v = jb.alpha * (double)__uint_as_float(r[q]);
          cc[gm] = (jb.beta == 0.0) ? v : fma(jb.beta, cc[gm], v);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(kTcN));
  if (tid == 0) {
    if (!ok) atomicCAS(status, 0, -7);
    else {
      const int mt = min(kTcM, jb.M - m0), nt = min(kTcN, jb.N - n0);
      add_work(status, kind, 2.0 * jb.K * mt * nt, 8.0 * ((double)mt * nt + (double)(mt + nt) * jb.K));
    }
  }
}

int launch_wait_selftest(long long limit, int* status, cudaStream_t s) {
  k_wait_selftest<<<1, 64, 0, s>>>(limit, status);
  return (int)cudaGetLastError();
}

long long tc_wait_limit() { return kTcWaitLimit; }

int launch_gemm_tc3(const GemmJob* jobs, int njobs, int max_m, int max_n, int aligned16, int* status, int kind,
                    cudaStream_t s) {
  if (njobs <= 0) return 0;
  const size_t sm = (size_t)kTcStages * kTcStageBytes + 1024;
  dim3 grid((unsigned)((max_n + kTcN - 1) / kTcN), (unsigned)((max_m + kTcM - 1) / kTcM), (unsigned)njobs);
  if (aligned16) {
    cudaFuncSetAttribute(k_gemm_tc3<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_gemm_tc3<2><<<grid, kTcThreads, sm, s>>>(jobs, status, kind);
  } else {
    cudaFuncSetAttribute(k_gemm_tc3<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_gemm_tc3<1><<<grid, kTcThreads, sm, s>>>(jobs, status, kind);
  }
  return (int)cudaGetLastError();
}

}  // namespace tlr
