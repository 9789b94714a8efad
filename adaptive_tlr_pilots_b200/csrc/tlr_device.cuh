// Device-side building blocks shared by the TLR kernels (sm_100a, FP64).
//
// Everything here is cooperative at the CTA level unless named warp_*.  Routines take
// generic pointers so the same code runs on shared or global (L2-resident) operands.
// All reductions are deterministic (fixed shuffle/shared-memory order): a log-likelihood
// evaluated twice on the same inputs is bit-identical.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef TLR_RESTRICT
#define TLR_RESTRICT __restrict__
#endif

namespace tlr {

constexpr double kSqrt3 = 1.7320508075688772935;
constexpr double kSqrt5 = 2.2360679774997896964;

// ---------------------------------------------------------------- FP64 tensor cores, async copies
// D = A B + D on the FP64 tensor cores, one 8 x 8 x 4 step per warp (g = lane / 4, t = lane % 4):
// a = A[g][t], b = B[t][g], d0 = D[g][2t], d1 = D[g][2t + 1].  Exact FP64 fused multiply-adds.
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// 16-byte global -> shared copy that completes asynchronously; bytes beyond src_bytes are zero.
// Both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum over the CTA; every thread gets the result.  `red` needs 33 doubles of shared memory.
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    double s = lane < nw ? red[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) red[32] = s;
  }
  __syncthreads();
  return red[32];
}

// ---------------------------------------------------------------- work counters
// The plan's control block: int status, three ints of padding, then [flops, bytes] doubles per
// kernel kind (algorithmic counts, accumulated by the kernels for the roofline report).
__device__ __forceinline__ void add_work(const int* status, int kind, double flops, double bytes) {
  double* w = reinterpret_cast<double*>(const_cast<int*>(status) + 4);
  atomicAdd(w + 2 * kind, flops);
  atomicAdd(w + 2 * kind + 1, bytes);
}

// ---------------------------------------------------------------- covariance model
// Matern kernel sigma2 k(h): nu = 3/2, k = (1 + x) e^{-x}, x = sqrt(3) h / range
// (codes/11_tlr_rank_rules.py:35-37 with the sigma2 scaling of codes/17_tlr_cholesky_pilot.py:161);
// nu = 5/2 (nu5 != 0), k = (1 + x + x^2 / 3) e^{-x}, x = sqrt(5) h / range
// (codes/24_screening_stress.py:30-43, the kernel it patches in for the regime sweeps).
__device__ __forceinline__ double matern_cov(double ax, double ay, double bx, double by, double sigma2,
                                             double inv_range, int nu5) {
  const double dx = ax - bx, dy = ay - by;
  const double h = sqrt(fmax(dx * dx + dy * dy, 0.0));
  if (nu5) {
    const double x = kSqrt5 * h * inv_range;
    return sigma2 * ((1.0 + x + x * x / 3.0) * exp(-x));
  }
  const double x = kSqrt3 * h * inv_range;
  return sigma2 * ((1.0 + x) * exp(-x));
}

// ---------------------------------------------------------------- rank rule
// sig[0..m) sorted descending; extra2 = squared norm of what lies outside the represented
// subspace.  tail[r] = sqrt(extra2 + sum_{t>=r} sig_t^2) accumulated from the smallest
// value up (codes/17_tlr_cholesky_pilot.py:113).  Returns the smallest r with tail[r] <= thr,
// or -1 when even tail[m] > thr.  Single thread.
__device__ __forceinline__ int select_rank(const double* sig, int m, double extra2, double thr,
                                           double* tail_at_rank) {
  double acc = extra2;
  int r = (sqrt(acc) <= thr) ? m : -1;
  double tr = sqrt(acc);
  for (int t = m - 1; t >= 0; --t) {
    acc += sig[t] * sig[t];
    const double tl = sqrt(acc);
    if (tl <= thr) { r = t; tr = tl; }
  }
  if (tail_at_rank) *tail_at_rank = tr;
  return r;
}

// ---------------------------------------------------------------- storage precision (rule 'mixed')
// x rounded to p-bit storage as the reference simulates it (codes/17_tlr_cholesky_pilot.py:41-55):
// p = 32 / 16 an IEEE cast with round-to-nearest-even (numpy's astype), p = 8 |x| = m 2^e with
// e = floor(log2 |x|) clipped to [-9, 8] and m rounded to 3 fraction bits (half to even), at most
// 448.  The exponent is read exactly with frexp; where numpy's floor(log2) lands one higher (|x|
// just below a power of two) both roundings give the same power of two.
__device__ __forceinline__ double round_bits(double x, int p) {
  if (p == 32) return (double)__double2float_rn(x);
  if (p == 16) return (double)__half2float(__double2half(x));
  if (p == 8) {
    const double a = fabs(x);
    if (a == 0.0) return 0.0;
    int ex;
    frexp(a, &ex);
    const int e = min(max(ex - 1, -9), 8);
    const double v = fmin(rint(ldexp(a, -e) * 8.0) / 8.0 * ldexp(1.0, e), 448.0);
    return copysign(v, x);
  }
  return x;
}

// A factor entry as stored in p bits (17:58-66): for p < 32 scaled so that the factor's largest
// magnitude `top` maps to half the format's largest value (224 FP8, 32752 FP16), rounded, unscaled.
__device__ __forceinline__ double store_entry(double x, int p, double top) {
  if (p == 64 || top == 0.0) return x;
  if (p == 32) return round_bits(x, 32);
  const double scale = (p == 8 ? 224.0 : 32752.0) / top;
  return round_bits(x * scale, p) / scale;
}

// Maximum over the CTA; every thread gets the result.  `red` needs 33 doubles of shared memory.
__device__ __forceinline__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    double m = lane < nw ? red[lane] : 0.0;
    m = warp_max(m);
    if (lane == 0) red[32] = m;
  }
  __syncthreads();
  return red[32];
}

// Store the pair (U: mu x r, V: mv x r, column-major, leading dimension ld) in the fewest bits
// p in {8, 16, 32} with ||U V^T - U~ V~^T||_F <= budget, else keep FP64 (17:69-82); U and V are
// rounded in place and p returned (every thread).  The error is formed from six r x r Gram
// products, ||E||^2 = <dU^T dU, V^T V> + 2 <dU^T U~, V^T dV> + <U~^T U~, dV^T dV> (E = dU V^T +
// U~ dV^T, dU = U - U~, dV = V - V~), whose terms are all of the size of the rounding error, so
// nothing large cancels.  `red` needs 33 doubles of shared memory.
// With forced in {8, 16, 32, 64} the search is skipped and that storage is used (replayed
// decisions); forced <= 0 searches.
__device__ inline int cta_round_pair(double* U, double* V, int mu, int mv, int r, int ld, double budget,
                                     double* red, int forced = 0) {
  if (r == 0) return 64;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  double mxu = 0.0, mxv = 0.0;
  for (int q = 0; q < r; ++q) {
    for (int a = tid; a < mu; a += blockDim.x) mxu = fmax(mxu, fabs(U[(size_t)q * ld + a]));
    for (int a = tid; a < mv; a += blockDim.x) mxv = fmax(mxv, fabs(V[(size_t)q * ld + a]));
  }
  const double topu = block_max(mxu, red);
  const double topv = block_max(mxv, red);
  int chosen = forced > 0 ? forced : 64;
  for (int p = 8; p <= 32 && forced <= 0; p *= 2) {
    // one warp per (c, d): the (c, d) entries of the six Gram products
    double part = 0.0;
    for (int e = warp; e < r * r; e += nwarp) {
      const int c = e % r, d = e / r;
      double g1 = 0.0, g2 = 0.0, g3 = 0.0, h1 = 0.0, h2 = 0.0, h3 = 0.0;
      const double* uc = U + (size_t)c * ld;
      const double* ud = U + (size_t)d * ld;
      const double* vc = V + (size_t)c * ld;
      const double* vd = V + (size_t)d * ld;
      for (int a = lane; a < mu; a += 32) {
        const double rc = store_entry(uc[a], p, topu), rd = store_entry(ud[a], p, topu);
        const double dc = uc[a] - rc, dd = ud[a] - rd;
        g1 = fma(dc, dd, g1);  // dU^T dU
        g2 = fma(dc, rd, g2);  // dU^T U~
        g3 = fma(rc, rd, g3);  // U~^T U~
      }
      for (int a = lane; a < mv; a += 32) {
        const double rd = store_entry(vd[a], p, topv);
        const double dc = vc[a] - store_entry(vc[a], p, topv), dd = vd[a] - rd;
        h1 = fma(vc[a], vd[a], h1);  // V^T V
        h2 = fma(vc[a], dd, h2);     // V^T dV
        h3 = fma(dc, dd, h3);        // dV^T dV
      }
      g1 = warp_sum(g1); g2 = warp_sum(g2); g3 = warp_sum(g3);
      h1 = warp_sum(h1); h2 = warp_sum(h2); h3 = warp_sum(h3);
      part += g1 * h1 + 2.0 * g2 * h2 + g3 * h3;
    }
    // every lane of a warp holds the warp's sum; count it once per warp
    const double err2 = block_sum(lane == 0 ? part : 0.0, red);
    if (sqrt(fmax(err2, 0.0)) <= budget) { chosen = p; break; }
  }
  if (chosen < 64) {
    for (int q = 0; q < r; ++q) {
      for (int a = tid; a < mu; a += blockDim.x) U[(size_t)q * ld + a] = store_entry(U[(size_t)q * ld + a], chosen, topu);
      for (int a = tid; a < mv; a += blockDim.x) V[(size_t)q * ld + a] = store_entry(V[(size_t)q * ld + a], chosen, topv);
    }
  }
  __syncthreads();
  return chosen;
}

// ---------------------------------------------------------------- Householder QR
// In-place Householder QR of the m x n column-major A (lda): R in the upper triangle,
// reflector vectors below the diagonal (implicit unit leading entry), tau[0..n).
// Same reflector convention as LAPACK dgeqr2/dlarfg.  One warp per trailing column.
// block_sum's value without its broadcast barrier: every warp finishes the reduction itself (the
// same inputs through the same butterfly, so the same bits as block_sum).  The leading barrier,
// which orders this call's writes of red[0..warps) after earlier readers, may be skipped (lead =
// false, uniform over the CTA) when every thread has passed a barrier since its last read of red.
__device__ __forceinline__ double block_sum_nb(double v, double* red, bool lead) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  if (lead) __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  return warp_sum(lane < nw ? red[lane] : 0.0);
}

__device__ inline void cta_geqr2(double* A, int lda, int m, int n, double* tau, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int kmax = n < m ? n : m;
  for (int c = 0; c < kmax; ++c) {
    double* col = A + (size_t)c * lda;
    double s = 0.0;
    for (int t = c + 1 + threadIdx.x; t < m; t += blockDim.x) { const double x = col[t]; s += x * x; }
    // columns after the first: the previous column's two barriers follow every read of red
    const double sig2 = block_sum_nb(s, red, c == 0);
    const double alpha = col[c];
    double beta, tc, scale;
    if (sig2 == 0.0) { tc = 0.0; beta = alpha; scale = 1.0; }
    else {
      beta = -copysign(sqrt(alpha * alpha + sig2), alpha);
      tc = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    if (tc != 0.0)
      for (int t = c + 1 + threadIdx.x; t < m; t += blockDim.x) col[t] *= scale;
    __syncthreads();
    // every thread has read alpha; the updates below read only col[t > c]
    if (threadIdx.x == 0) { col[c] = beta; tau[c] = tc; }
    for (int j = c + 1 + warp; j < n; j += nwarp) {
      double* aj = A + (size_t)j * lda;
      double w = 0.0;
      for (int t = c + 1 + lane; t < m; t += 32) w += col[t] * aj[t];
      w = (warp_sum(w) + aj[c]) * tc;
      for (int t = c + 1 + lane; t < m; t += 32) aj[t] -= w * col[t];
      __syncwarp();
      if (lane == 0) aj[c] -= w;
    }
    __syncthreads();
  }
  for (int c = kmax + threadIdx.x; c < n; c += blockDim.x) tau[c] = 0.0;
  __syncthreads();
}

// The R of cta_geqr2, bit for bit, when neither the reflectors nor tau are wanted: on return the
// entries of A on and above the diagonal hold R, those below it are left as they were.  The
// reflector is applied as column x 1 / (alpha - beta), the very product cta_geqr2 stores (scale is
// 1 exactly when tau is 0), so no scaling pass and its barrier.  With m <= 32 only warp 0 holds
// entries of a column norm, so block_sum's value is warp 0's butterfly: every warp forms that itself
// and a column costs one barrier.
__device__ inline void cta_geqr2_r(double* A, int lda, int m, int n, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int kmax = n < m ? n : m;
  for (int c = 0; c < kmax; ++c) {
    double* col = A + (size_t)c * lda;
    double sig2;
    if (m <= 32) {
      const int t = c + 1 + lane;
      const double x = t < m ? col[t] : 0.0;
      sig2 = warp_sum(x * x);
    } else {
      double s = 0.0;
      for (int t = c + 1 + threadIdx.x; t < m; t += blockDim.x) { const double x = col[t]; s += x * x; }
      sig2 = block_sum_nb(s, red, c == 0);  // later columns: the barrier below follows every read of red
    }
    const double alpha = col[c];
    double beta, tc, scale;
    if (sig2 == 0.0) { tc = 0.0; beta = alpha; scale = 1.0; }
    else {
      beta = -copysign(sqrt(alpha * alpha + sig2), alpha);
      tc = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    for (int j = c + 1 + warp; j < n; j += nwarp) {
      double* aj = A + (size_t)j * lda;
      double w = 0.0;
      for (int t = c + 1 + lane; t < m; t += 32) {
        const double v = col[t] * scale;
        w += v * aj[t];
      }
      w = (warp_sum(w) + aj[c]) * tc;
      for (int t = c + 1 + lane; t < m; t += 32) {
        const double v = col[t] * scale;
        aj[t] -= w * v;
      }
      __syncwarp();
      if (lane == 0) aj[c] -= w;
    }
    __syncthreads();
    // every thread has read alpha; no later column reads this entry
    if (threadIdx.x == 0) col[c] = beta;
  }
  __syncthreads();
}

// Copy the upper-triangular R (n x n, or kmax rows) out of a factored A into Rout (ldr),
// zeroing the strictly lower part.
__device__ inline void cta_copy_r(const double* A, int lda, int m, int n, double* R, int ldr) {
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    R[(size_t)j * ldr + i] = (i <= j && i < m) ? A[(size_t)j * lda + i] : 0.0;
  }
  __syncthreads();
}

// Overwrite the factored A (reflectors + tau from cta_geqr2) with the explicit m x n Q
// (LAPACK dorg2r order: backward accumulation).
__device__ inline void cta_org2r(double* A, int lda, int m, int n, const double* tau) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int kmax = n < m ? n : m;
  // columns beyond min(m, n) (only when n > m, not used here) become unit columns
  for (int c = kmax - 1; c >= 0; --c) {
    const double* v = A + (size_t)c * lda;
    const double tc = tau[c];
    if (c < n - 1 && tc != 0.0) {
      for (int j = c + 1 + warp; j < n; j += nwarp) {
        double* aj = A + (size_t)j * lda;
        double w = 0.0;
        for (int t = c + 1 + lane; t < m; t += 32) w += v[t] * aj[t];
        w = (warp_sum(w) + aj[c]) * tc;
        for (int t = c + 1 + lane; t < m; t += 32) aj[t] -= w * v[t];
        __syncwarp();
        if (lane == 0) aj[c] -= w;
      }
    }
    __syncthreads();
    double* ac = A + (size_t)c * lda;
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
      if (t < c) ac[t] = 0.0;
      else if (t == c) ac[t] = 1.0 - tc;
      else ac[t] = -tc * ac[t];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- one-sided Jacobi SVD
// Hestenes one-sided Jacobi on the m x n column-major M (ldm): on return M <- M V has
// mutually orthogonal columns, V (n x n, ldv; NULL: not formed) holds the right singular vectors, sig[c] the
// column norms (singular values, unsorted) and perm[0..n) the column order by descending
// singular value (ties by index).  Round-robin parallel ordering, one warp per pair; squared
// column norms are computed afresh at the start of every sweep and updated by the rotation
// formulas within it (a_pp' = a_pp - t a_pq, a_qq' = a_qq + t a_pq), so a pair costs one inner
// product.  `sig` needs n doubles, `iflag` two ints of shared memory.  Returns the sweeps used.
// With floor_rel > 0, a column whose squared norm is at most floor_rel times the largest squared
// column norm counts as zero and is not rotated: columns at the rounding level of the others
// (from cores assembled out of Gram matrices) would otherwise keep the relative test of their
// pairs failing forever.
__device__ inline int cta_jacobi_svd(double* M, int ldm, int m, int n, double* V, int ldv, double* sig,
                                     int* perm, int* iflag, int max_sweeps = 40, double floor_rel = 0.0) {
  // largest squared column norm of a sweep, as the bits of a double >= 0 (their integer order is
  // the doubles' order); two slots, alternating like the flags
  __shared__ unsigned long long s_mx[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  if (V)
    for (int j = warp; j < n; j += nwarp)
      for (int i = lane; i < n; i += 32) V[(size_t)j * ldv + i] = (i == j) ? 1.0 : 0.0;
  const int np = (n + 1) & ~1;  // even number of players (one dummy when n is odd)
  // rotate unless the pair is orthogonal to working precision, |cos| <= m eps (the singular
  // values then carry a relative error of order cos^2)
  const double tol = (double)(m > 4 ? m : 4) * 2.220446049250313e-16;
  const double tol2 = tol * tol;
  int sweep = 0;
  if (n > 1) {
    // two flags, alternating: the flag of sweep s + 1 is cleared during sweep s, after the barrier
    // that follows every read of it at the end of sweep s - 1
    if (threadIdx.x == 0) {
      iflag[0] = 0;
      s_mx[0] = 0ull;
    }
    __syncthreads();
    for (sweep = 0; sweep < max_sweeps; ++sweep) {
      for (int c = warp; c < n; c += nwarp) {
        const double* mc = M + (size_t)c * ldm;
        double a = 0.0;
        for (int t = lane; t < m; t += 32) a += mc[t] * mc[t];
        a = warp_sum(a);
        if (lane == 0) {
          sig[c] = a;
          if (floor_rel > 0.0) atomicMax(&s_mx[sweep & 1], (unsigned long long)__double_as_longlong(a));
        }
      }
      __syncthreads();  // the column norms above come from every warp
      if (threadIdx.x == 0) {
        iflag[(sweep + 1) & 1] = 0;
        s_mx[(sweep + 1) & 1] = 0ull;
      }
      const double floor2 = floor_rel * __longlong_as_double((long long)s_mx[sweep & 1]);
      for (int round = 0; round < np - 1; ++round) {
        for (int pr = warp; pr < np / 2; pr += nwarp) {
          // circle method: player 0 fixed, the others rotate
          const int a = (pr == 0) ? 0 : 1 + ((pr - 1 + round) % (np - 1));
          const int b = 1 + ((np - 2 - pr + round) % (np - 1));
          if (a >= n || b >= n) continue;
          const int p = a < b ? a : b, q = a < b ? b : a;
          double* mp = M + (size_t)p * ldm;
          double* mq = M + (size_t)q * ldm;
          double apq = 0.0;
          for (int t = lane; t < m; t += 32) apq += mp[t] * mq[t];
          apq = warp_sum(apq);
          const double app = sig[p], aqq = sig[q];
          if (apq != 0.0 && apq * apq > tol2 * app * aqq && fmin(app, aqq) > floor2) {
            // t = tan of the rotation angle, the smaller root of t^2 + 2 zeta t - 1 = 0 with
            // zeta = (a_qq - a_pp) / (2 a_pq); for |zeta| > 1e7, t = 1 / (2 zeta) to full precision
            const double d = aqq - app;
            double t;
            if (fabs(d) > 2.0e7 * fabs(apq)) t = apq / d;
            else {
              const double zeta = 0.5 * d / apq;
              t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            }
            const double cs = rsqrt(1.0 + t * t), sn = cs * t;
            for (int r = lane; r < m; r += 32) {
              const double x = mp[r], y = mq[r];
              mp[r] = cs * x - sn * y;
              mq[r] = sn * x + cs * y;
            }
            if (V) {
              double* vp = V + (size_t)p * ldv;
              double* vq = V + (size_t)q * ldv;
              for (int r = lane; r < n; r += 32) {
                const double x = vp[r], y = vq[r];
                vp[r] = cs * x - sn * y;
                vq[r] = sn * x + cs * y;
              }
            }
            __syncwarp();
            if (lane == 0) {
              sig[p] = app - t * apq;
              sig[q] = aqq + t * apq;
              iflag[sweep & 1] = 1;
            }
          }
        }
        __syncthreads();
      }
      if (!iflag[sweep & 1]) break;
    }
  }
  // singular values = column norms
  for (int c = warp; c < n; c += nwarp) {
    const double* mc = M + (size_t)c * ldm;
    double s = 0.0;
    for (int t = lane; t < m; t += 32) s += mc[t] * mc[t];
    s = warp_sum(s);
    if (lane == 0) sig[c] = sqrt(s);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const double sc = sig[c];
    int pos = 0;
    for (int d = 0; d < n; ++d) {
      const double sd = sig[d];
      pos += (sd > sc) || (sd == sc && d < c);
    }
    perm[pos] = c;
  }
  __syncthreads();
  return sweep;
}

}  // namespace tlr
