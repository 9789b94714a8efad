// Tensor-core (tcgen05) GEMM for the mixed-precision path: C = alpha op(A) op(B) + beta C with FP64
// operands and result, products formed on the 5th-generation tensor cores as split TF32
// ("3xTF32": x = hi + lo with hi, lo TF32, A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi) accumulated in
// FP32 in tensor memory.  Relative accuracy is that of FP32 (about 1e-7 per product), which keeps
// the selected-inversion gradient within ~1e-5 of the FP64 one (single-pass TF32 loses ~1e-2 on
// the range component).
//
// Two kernels per batch of GEMM jobs.  k_split_tf32 converts each distinct operand once: rows x K
// of FP64 into zero-padded blocks of 128 rows x 16 k, block (row tile t, K slice s) stored
// contiguously at (t * nks + s) x 16 KB as hi TF32 then lo TF32, each in the canonical K-major,
// no-swizzle UMMA layout (core matrices of 8 rows x 16 bytes; rows of a core matrix 16 B apart,
// 8-row groups 128 B apart, the two 16-byte K halves of one MMA 2048 B apart).  A block is then
// exactly the shared-memory image of one operand's slice.  k_gemm_tc3 computes a 128 x 128 output
// tile per CTA (accumulator: 128 TMEM lanes x 128 columns; two CTAs per SM) with two single-thread
// roles over a ring of three 32 KB stages: a producer thread moves each slice's A and B blocks with two bulk async
// copies (cp.async.bulk, completing on the stage's "full" mbarrier with a byte count), and an MMA
// thread waits on "full", issues 2 K-steps x 3 tcgen05.mma.kind::tf32 and commits them to the
// stage's "empty" mbarrier, which releases the stage to the producer.  The other warps join for
// the epilogue (tcgen05.ld of the accumulator, alpha / beta, column scatter).  The MMA sequence
// (K-steps of 8 in order, three products each) is fixed, so results do not depend on the staging.
// Waits are bounded: on timeout the kernel sets an error status, waits (bounded) for its copies
// in flight, frees its tensor memory and returns.
#include <stdint.h>

#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace tlr {

constexpr int kTcM = 128;
constexpr int kTcN = 128;
constexpr int kTcBK = 16;                               // k per slice: two MMA K-steps
constexpr int kTcStages = 3;                            // two CTAs per SM: one's epilogue overlaps the other's MMAs
constexpr int kTcThreads = 256;                         // warp 0: copies, warp 1: MMAs, all: epilogue
constexpr int kTcBlockFloats = 2 * kTcM * kTcBK;        // one operand block: hi + lo, 16 KB
constexpr int kTcOpBytes = kTcBlockFloats * 4;
constexpr int kTcStageBytes = 2 * kTcOpBytes;           // A block, then B block
constexpr int kSplitThreads = 256;
constexpr int kSplitPer = 4;                            // blocks per CTA of the split
static_assert(kTcM == kTcN && kTcBK == 16, "block layout assumes 128-row tiles and 16-k slices");
static_assert(2 * (kTcStageBytes * kTcStages + 2048) <= 228 * 1024, "two CTAs per SM exceed shared memory");
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

// One CTA per kSplitPer consecutive blocks (128 rows x 16 k) of an operand: blockIdx.y the
// operand, blockIdx.x the group of blocks.  Thread (r = tid % 128, g = tid / 128 + 2i) handles k
// values 4g .. 4g + 3 of tile row r in each block; every load of the group is issued before the
// first conversion, so a thread keeps 32 loads in flight.
__global__ void __launch_bounds__(kSplitThreads) k_split_tf32(const SplitJob* TLR_RESTRICT jobs,
                                                            int* TLR_RESTRICT status, int kind) {
  if (*status != 0) return;
  const SplitJob j = jobs[blockIdx.y];
  const int nks = (j.K + kTcBK - 1) / kTcBK;
  const int nblk = ((j.rows + kTcM - 1) / kTcM) * nks;
  const int blk0 = (int)blockIdx.x * kSplitPer;
  if (blk0 >= nblk) return;
  const int r = threadIdx.x & (kTcM - 1), g0 = threadIdx.x >> 7;
  constexpr int kG = kTcBK / 4 / (kSplitThreads / kTcM);  // k groups per thread and block: 2
  double x[kSplitPer][kG][4];
#pragma unroll
  for (int b = 0; b < kSplitPer; ++b) {
    const int blk = blk0 + b;
    const int gr = (blk / nks) * kTcM + r, k0 = (blk % nks) * kTcBK;
#pragma unroll
    for (int i = 0; i < kG; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int gk = k0 + 4 * (g0 + 2 * i) + c;
        x[b][i][c] = (blk < nblk && gr < j.rows && gk < j.K)
                         ? (j.kcont ? j.src[(size_t)gr * j.ld + gk] : j.src[(size_t)gk * j.ld + gr])
                         : 0.0;
      }
  }
#pragma unroll
  for (int b = 0; b < kSplitPer; ++b) {
    if (blk0 + b >= nblk) break;
    float* out = j.dst + (size_t)(blk0 + b) * kTcBlockFloats;
#pragma unroll
    for (int i = 0; i < kG; ++i) tc_write4(out, x[b][i], r, g0 + 2 * i);
  }
  if (threadIdx.x == 0) {
    double bytes = 0.0;
    for (int b = 0; b < kSplitPer && blk0 + b < nblk; ++b) {
      const int blk = blk0 + b;
      const int mt = min(kTcM, j.rows - (blk / nks) * kTcM), kt = min(kTcBK, j.K - (blk % nks) * kTcBK);
      bytes += 8.0 * mt * kt + 4.0 * kTcBlockFloats;
    }
    add_work(status, kind, 0.0, bytes);
  }
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// contiguous global -> shared bulk copy (16-byte aligned, size a multiple of 16) that completes
// `bytes` of the transaction count of `mbar`
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 2) k_gemm_tc3(const GemmJob* TLR_RESTRICT jobs,
                                                 const TcOperands* TLR_RESTRICT ops, int* TLR_RESTRICT status,
                                                 int kind) {
  if (*status != 0) return;
  const GemmJob jb = jobs[blockIdx.z];
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
  if (m0 >= jb.M || n0 >= jb.N) return;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t full[kTcStages], empty[kTcStages];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int timed_out, issued, committed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(kTcN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
    timed_out = 0;
    issued = 0;
    committed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem_d = tmem_base_sh;
  const int nk = (jb.K + kTcBK - 1) / kTcBK;
  const uint32_t sbase = smem_u32(tc_smem);
  if (nk > 0 && tid == 0) {
    // producer: slice s into stage s % 3 once the MMAs of slice s - 3 have released it
    const TcOperands op = ops[blockIdx.z];
    const float* pa = op.a + (size_t)(m0 / kTcM) * nk * kTcBlockFloats;
    const float* pb = op.b + (size_t)(n0 / kTcN) * nk * kTcBlockFloats;
    int s = 0;
    for (; s < nk; ++s) {
      const int st = s % kTcStages;
      if (s >= kTcStages && !mbar_wait(smem_u32(&empty[st]), (uint32_t)((s / kTcStages - 1) & 1))) {
        timed_out = 1;
        break;
      }
      const uint32_t fb = smem_u32(&full[st]);
      mbar_expect_tx(fb, kTcStageBytes);
      bulk_g2s(sbase + st * kTcStageBytes, pa + (size_t)s * kTcBlockFloats, kTcOpBytes, fb);
      bulk_g2s(sbase + st * kTcStageBytes + kTcOpBytes, pb + (size_t)s * kTcBlockFloats, kTcOpBytes, fb);
    }
    issued = s;
  } else if (nk > 0 && tid == 32) {
    // MMA issuer
    const uint32_t idesc = umma_idesc_tf32(kTcM, kTcN);
    const uint32_t lbo = kTcM * 16, sbo = 128;
    int s = 0;
    for (; s < nk; ++s) {
      const int st = s % kTcStages;
      if (!mbar_wait(smem_u32(&full[st]), (uint32_t)((s / kTcStages) & 1))) {
        timed_out = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t aH = sbase + st * kTcStageBytes, aL = aH + kTcM * kTcBK * 4;
      const uint32_t bH = aH + kTcOpBytes, bL = bH + kTcN * kTcBK * 4;
#pragma unroll
      for (int ks = 0; ks < kTcBK / 8; ++ks) {
        const uint32_t o = ks * 2 * kTcM * 16;
        const uint64_t dAh = umma_desc(aH + o, lbo, sbo), dAl = umma_desc(aL + o, lbo, sbo);
        const uint64_t dBh = umma_desc(bH + o, lbo, sbo), dBl = umma_desc(bL + o, lbo, sbo);
        const uint32_t first = (s == 0 && ks == 0) ? 0u : 1u;
        mma_tf32(tmem_d, dAh, dBh, idesc, first);
        mma_tf32(tmem_d, dAh, dBl, idesc, 1u);
        mma_tf32(tmem_d, dAl, dBh, idesc, 1u);
      }
      mma_commit(smem_u32(&empty[st]));
    }
    committed = s;
  }
  __syncwarp();
  __syncthreads();
  if (tid == 0 && nk > 0) {
    if (!timed_out) {
      // the last commit covers every MMA issued before it
      const int last = nk - 1;
      if (!mbar_wait(smem_u32(&empty[last % kTcStages]), (uint32_t)((last / kTcStages) & 1))) timed_out = 1;
    } else {
      // failure: let the copies in flight land (the last slices issued, one per stage), and the
      // MMAs already issued finish (their last commit), before the tensor memory is released
      for (int q = max(0, issued - kTcStages); q < issued; ++q)
        mbar_wait(smem_u32(&full[q % kTcStages]), (uint32_t)((q / kTcStages) & 1));
      if (committed > 0) {
        const int last = committed - 1;
        mbar_wait(smem_u32(&empty[last % kTcStages]), (uint32_t)((last / kTcStages) & 1));
      }
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const bool ok = !timed_out;
  if (ok) {
    // warp w reads TMEM lane quarter w % 4 (the lanes a warp may access) and column half w / 4
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

int launch_split_tf32(const SplitJob* jobs, int njobs, int max_blocks, int* status, int kind, cudaStream_t s) {
  if (njobs <= 0 || max_blocks <= 0) return 0;
  const unsigned gx = (unsigned)((max_blocks + kSplitPer - 1) / kSplitPer);
  k_split_tf32<<<dim3(gx, (unsigned)njobs), kSplitThreads, 0, s>>>(jobs, status, kind);
  return (int)cudaGetLastError();
}

int launch_gemm_tc3(const GemmJob* jobs, const TcOperands* ops, int njobs, int max_m, int max_n, int* status, int kind,
                    cudaStream_t s) {
  if (njobs <= 0) return 0;
  const size_t sm = (size_t)kTcStages * kTcStageBytes + 1024;
  cudaFuncSetAttribute(k_gemm_tc3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 grid((unsigned)((max_n + kTcN - 1) / kTcN), (unsigned)((max_m + kTcM - 1) / kTcM), (unsigned)njobs);
  k_gemm_tc3<<<grid, kTcThreads, sm, s>>>(jobs, ops, status, kind);
  return (int)cudaGetLastError();
}

size_t tc_panel_floats(int rows, int K) {
  return (size_t)((rows + kTcM - 1) / kTcM) * ((K + kTcBK - 1) / kTcBK) * kTcBlockFloats;
}
int tc_panel_blocks(int rows, int K) { return ((rows + kTcM - 1) / kTcM) * ((K + kTcBK - 1) / kTcBK); }

}  // namespace tlr
