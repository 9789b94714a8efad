// Tensor-core (tcgen05) GEMM for the mixed-precision path: C = alpha op(A) op(B) + beta C with FP64
// operands and result, products formed on the 5th-generation tensor cores as split TF32
// ("3xTF32": x = hi + lo with hi, lo TF32, A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi) accumulated in
// FP32 in tensor memory.  Relative accuracy is that of FP32 (about 1e-7 per product), which keeps
// the selected-inversion gradient within ~1e-5 of the FP64 one (single-pass TF32 loses ~1e-2 on
// the range component).
//
// One CTA of 512 threads (four per row of the tile, so that sixteen warps share the conversion
// latency) computes a 128 x N_TILE output tile (N_TILE = 128): the accumulator is
// 128 TMEM lanes x 128 columns.  K advances in slices of 32: every thread converts and splits its
// share of the FP64 slice into shared memory in the canonical K-major, no-swizzle UMMA layout
// (core matrices of 8 rows x 16 bytes; rows of a core matrix 16 B apart, 8-row groups 128 B
// apart, the two 16-byte K halves of one MMA 2048 B apart for A), fences the generic-proxy writes
// for the async proxy, and thread 0 issues 4 K-steps x 3 tcgen05.mma.kind::tf32 and commits them
// to the stage's mbarrier.  Two stages alternate, so the conversion of slice s+1 overlaps the MMAs
// of slice s, and the global loads of slice s+1 are issued (into a second register set) before
// slice s is converted, so their latency overlaps that work.  Waits on the mbarriers are bounded: on timeout the kernel sets an error status,
// frees its tensor memory and returns.
#include <stdint.h>

#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace tlr {

constexpr int kTcM = 128;
constexpr int kTcN = 128;
constexpr int kTcBK = 32;
constexpr int kTcStages = 2;
constexpr int kTcThreads = 512;                   // 4 threads per row of a 128-row slice
constexpr int kTcPerThread = kTcBK * 2 / (kTcThreads / kTcM) / 2;  // k values of A (and of B) per thread: 8
// bytes per stage: A_hi, A_lo (128 x 32 x 4), B_hi, B_lo (128 x 32 x 4)
constexpr int kTcStageBytes = 4 * kTcM * kTcBK * 4;
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
  int fail = 0;
  // global -> registers for slice `it`: thread -> (row r = tid / 4, K groups (tid & 3) * 2 .. + 1
  // of 4 consecutive k each), all 8 loads of A and of B issued before any of them is used
  auto gload = [&](int it, double (&va)[kTcPerThread], double (&vb)[kTcPerThread]) {
    const int k0 = it * kTcBK;
    const int r = tid >> 2, gh = (tid & 3) * 2;
    const int gma = m0 + r, gnb = n0 + r;
#pragma unroll
    for (int q = 0; q < kTcPerThread; ++q) {
      const int gk = k0 + gh * 4 + q;
      va[q] = (gma < jb.M && gk < jb.K)
                  ? (jb.transA ? jb.A[(size_t)gma * jb.lda + gk] : jb.A[(size_t)gk * jb.lda + gma])
                  : 0.0;
      vb[q] = (gnb < jb.N && gk < jb.K)
                  ? (jb.transB ? jb.B[(size_t)gk * jb.ldb + gnb] : jb.B[(size_t)gnb * jb.ldb + gk])
                  : 0.0;
    }
  };
  // registers of slice `it` -> its shared-memory stage (split TF32, each group of 4 as one 16-byte
  // store), then thread 0 issues the slice's MMAs; false (in every thread) on a timed-out wait
  auto stage_in = [&](int it, const double (&va)[kTcPerThread], const double (&vb)[kTcPerThread]) -> bool {
    const int st = it & 1;
    unsigned char* sbase = tc_smem + st * kTcStageBytes;
    float* Ahi = reinterpret_cast<float*>(sbase);
    float* Alo = Ahi + kTcM * kTcBK;
    float* Bhi = Alo + kTcM * kTcBK;
    float* Blo = Bhi + kTcN * kTcBK;
    int bad = 0;
    if (it >= kTcStages) {
      // the MMAs that read this stage two slices ago must be done before it is overwritten
      if (!mbar_wait(smem_u32(&mbar[st]), (uint32_t)(((it - kTcStages) >> 1) & 1))) bad = 1;
    }
    if (__syncthreads_or(bad)) return false;
    {
      const int r = tid >> 2, gh = (tid & 3) * 2;
#pragma unroll
      for (int g = 0; g < kTcPerThread / 4; ++g) {
        float4 ah, al, bh, bl;
        float* pah = &ah.x; float* pal = &al.x; float* pbh = &bh.x; float* pbl = &bl.x;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float fa = (float)va[4 * g + c], fb = (float)vb[4 * g + c];
          const uint32_t ha = to_tf32(fa), hb = to_tf32(fb);
          pah[c] = __uint_as_float(ha);
          pal[c] = __uint_as_float(to_tf32(fa - __uint_as_float(ha)));
          pbh[c] = __uint_as_float(hb);
          pbl[c] = __uint_as_float(to_tf32(fb - __uint_as_float(hb)));
        }
        const int chunk = gh + g;
        *reinterpret_cast<float4*>(Ahi + chunk * (kTcM * 4) + r * 4) = ah;
        *reinterpret_cast<float4*>(Alo + chunk * (kTcM * 4) + r * 4) = al;
        *reinterpret_cast<float4*>(Bhi + chunk * (kTcN * 4) + r * 4) = bh;
        *reinterpret_cast<float4*>(Blo + chunk * (kTcN * 4) + r * 4) = bl;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t aH = smem_u32(Ahi), aL = smem_u32(Alo), bH = smem_u32(Bhi), bL = smem_u32(Blo);
      const uint32_t lboA = kTcM * 16, lboB = kTcN * 16, sbo = 128;
#pragma unroll
      for (int ks = 0; ks < kTcBK / 8; ++ks) {
        const uint32_t oa = ks * 2 * kTcM * 16, ob = ks * 2 * kTcN * 16;
        const uint64_t dAh = umma_desc(aH + oa, lboA, sbo), dAl = umma_desc(aL + oa, lboA, sbo);
        const uint64_t dBh = umma_desc(bH + ob, lboB, sbo), dBl = umma_desc(bL + ob, lboB, sbo);
        const uint32_t first = (it == 0 && ks == 0) ? 0u : 1u;
        mma_tf32(tmem_d, dAh, dBh, idesc, first);
        mma_tf32(tmem_d, dAh, dBl, idesc, 1u);
        mma_tf32(tmem_d, dAl, dBh, idesc, 1u);
      }
      mma_commit(smem_u32(&mbar[st]));
    }
    return true;
  };
  // two register sets: the loads of slice it + 1 are in flight while slice it is converted
  double a0[kTcPerThread], b0[kTcPerThread], a1[kTcPerThread], b1[kTcPerThread];
  if (nk > 0) gload(0, a0, b0);
  for (int it = 0; it < nk; it += 2) {
    if (it + 1 < nk) gload(it + 1, a1, b1);
    if (!stage_in(it, a0, b0)) {
      fail = 1;
      break;
    }
    if (it + 1 >= nk) break;
    if (it + 2 < nk) gload(it + 2, a0, b0);
    if (!stage_in(it + 1, a1, b1)) {
      fail = 1;
      break;
    }
  }
  // wait for the last commit (it covers every MMA issued before it)
  if (!fail && nk > 0 && tid == 0) {
    const int last = nk - 1;
    if (!mbar_wait(smem_u32(&mbar[last & 1]), (uint32_t)((last >> 1) & 1))) timed_out = 1;
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

int launch_gemm_tc3(const GemmJob* jobs, int njobs, int max_m, int max_n, int* status, int kind, cudaStream_t s) {
  if (njobs <= 0) return 0;
  const size_t sm = (size_t)kTcStages * kTcStageBytes + 1024;
  cudaFuncSetAttribute(k_gemm_tc3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 grid((unsigned)((max_n + kTcN - 1) / kTcN), (unsigned)((max_m + kTcM - 1) / kTcM), (unsigned)njobs);
  k_gemm_tc3<<<grid, kTcThreads, sm, s>>>(jobs, status, kind);
  return (int)cudaGetLastError();
}

}  // namespace tlr
