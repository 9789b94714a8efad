// Right-looking TLR Cholesky, forward solve and log-likelihood (FP64 parity path).
//
// Reference: codes/17_tlr_cholesky_pilot.py:168-205 (factorization), 230-240 (forward solve)
// and 259-266 (log-likelihood).  Per step k, in stream order:
//   k_diag_build(k)   A_kk = Sigma_kk - sum_{m<k} U_km (V_km^T V_km) U_km^T   (deferred updates,
//                     subtracted in the order m = 0, 1, ... of the reference's step-by-step updates)
//   k_potrf(k)        blocked Cholesky of A_kk (status k+1 when a pivot is not positive, as LAPACK
//                     potrf), log det partial, z_k = L_kk^{-1} rhs_k
//   k_trsm(k)         V_ik <- L_kk^{-1} V_ik for i > k; W_ik = V_ik^T V_ik; Y_ik = U_ik W_ik;
//                     rhs_i -= U_ik (V_ik^T z_k)
//   k_recompress(k)   A_ij <- truncate([U_ij, -U_ik W], [V_ij, U_jk]) for k < j < i, W = V_ik^T V_jk,
//                     skipped when r_ik = 0 or r_jk = 0 (17:189-194)
// Layout in HBM: diagonal tiles column-major (ld b); off-diagonal factors U, V column-major
// (ld b, cap columns per tile); tile (i, j), i > j, has index i (i - 1) / 2 + j.
#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace tlr {

__device__ __forceinline__ int tidx(int i, int j) { return i * (i - 1) / 2 + j; }

// ----------------------------------------------------------------------------------------
// A_kk = Sigma_kk - sum_{m<k} Y_km U_km^T, Y_km = U_km W_km (written by the panel solve of step m):
// the deferred diagonal updates as one product of inner dimension R_k = sum_m r_km.  One CTA per
// lower-triangular 32 x 32 block; the inner index runs over (m, q) in ascending order, 32 at a
// time through shared memory.
__global__ void __launch_bounds__(256) k_diag_build(const double* TLR_RESTRICT xy, int n, int b, int k,
                                                   const double* TLR_RESTRICT U, const double* TLR_RESTRICT Y,
                                                   const int* TLR_RESTRICT rank, int cap, double* TLR_RESTRICT D,
                                                   const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const EvalParams& prm = *eval_params(status);
  const double sigma2 = prm.sigma2, inv_range = prm.inv_range, nugget = prm.nugget;
  const int nu5 = prm.nu5;
  int blk = blockIdx.x, rb = 0;
  while (blk > rb) { blk -= rb + 1; ++rb; }
  const int cb = blk;
  const int bk = min(b, n - k * b);
  const int r0 = rb * 32, c0 = cb * 32;
  __shared__ int off[1025];
  __shared__ int cm[32], cq[32];
  __shared__ double Ya[32][33], Uc[32][33];
  const int tid = threadIdx.x, cl = tid & 31, rl = tid >> 5;
  if (tid == 0) {
    int o = 0;
    for (int m = 0; m < k; ++m) {
      off[m] = o;
      o += rank[tidx(k, m)];
    }
    off[k] = o;
    if (rb == 0 && cb == 0) add_work(status, 7, 0.5 * 2.0 * bk * bk * o, 4.0 * bk * bk);
  }
  double acc[4];
  const double2* p2 = reinterpret_cast<const double2*>(xy);
  const int cg = c0 + cl;
  const double2 pc = p2[k * b + min(cg, bk - 1)];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int ag = r0 + rl + 8 * q;
    const double2 pa = p2[k * b + min(ag, bk - 1)];
    acc[q] = matern_cov(pa.x, pa.y, pc.x, pc.y, sigma2, inv_range, nu5) + (ag == cg ? nugget : 0.0);
  }
  __syncthreads();
  const int R = off[k];
  for (int i0 = 0; i0 < R; i0 += 32) {
    if (tid < 32) {
      const int c = i0 + tid;
      int m = -1, q = 0;
      if (c < R) {
        int lo = 0, hi = k;  // off[lo] <= c < off[hi]
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (off[mid] <= c) lo = mid; else hi = mid;
        }
        m = lo;
        q = c - off[lo];
      }
      cm[tid] = m;
      cq[tid] = q;
    }
    __syncthreads();
    for (int e = tid; e < 32 * 32; e += 256) {
      const int rr = e & 31, cc = e >> 5;
      const int m = cm[cc];
      double ya = 0.0, uc = 0.0;
      if (m >= 0) {
        const size_t off_t = (size_t)tidx(k, m) * b * cap + (size_t)cq[cc] * b;
        if (r0 + rr < bk) ya = Y[off_t + r0 + rr];
        if (c0 + rr < bk) uc = U[off_t + c0 + rr];
      }
      Ya[rr][cc] = ya;
      Uc[rr][cc] = uc;
    }
    __syncthreads();
#pragma unroll 8
    for (int cc = 0; cc < 32; ++cc) {
      const double u = Uc[cl][cc];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(-Ya[rl + 8 * q][cc], u, acc[q]);
    }
    __syncthreads();
  }
  double* A = D + (size_t)k * b * b;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int ag = r0 + rl + 8 * q;
    if (ag < bk && cg < bk && ag >= cg) A[(size_t)cg * b + ag] = acc[q];
  }
}

// ----------------------------------------------------------------------------------------
// Panel solve for column k: one CTA per row tile i > k.
__global__ void __launch_bounds__(256) k_trsm(const double* TLR_RESTRICT D, int n, int b, int k, int nB,
                                             double* TLR_RESTRICT U, double* TLR_RESTRICT V,
                                             double* TLR_RESTRICT Wd, double* TLR_RESTRICT Y,
                                             const int* TLR_RESTRICT rank, int cap,
                                             const double* TLR_RESTRICT z, double* TLR_RESTRICT rhs,
                                             int* TLR_RESTRICT prec, int* TLR_RESTRICT blog_trsm, int prank,
                                             int pworld, const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const EvalParams& prm = *eval_params(status);
  const int round_store = prm.round_store, rmode = prm.rmode;
  const double thr_abs = prm.thr_abs;
  const int i = k + 1 + blockIdx.x;
  if (i >= nB || i % pworld != prank) return;  // block-row partition: this rank's rows only
  const int t = tidx(i, k);
  const int r = rank[t];
  if (r == 0) return;
  const int bk = min(b, n - k * b), bi = min(b, n - i * b);
  const double* L = D + (size_t)k * b * b;
  double* Vt = V + (size_t)t * b * cap;
  double* Ut = U + (size_t)t * b * cap;
  if (threadIdx.x == 0) add_work(status, 9, (double)bk * bk * r + 2.0 * bk * r * r + 4.0 * bk * r,
                                 8.0 * ((double)bk * bk * 0.5 + 2.0 * bk * r + bi * r));
  __shared__ double L11[32][33];
  __shared__ double dinv[32];
  __shared__ double Xp[32][65];
  __shared__ double zt[64];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int q0 = 0; q0 < r; q0 += 64) {
    const int rq = min(64, r - q0);
    for (int p0 = 0; p0 < bk; p0 += 32) {
      const int pw = min(32, bk - p0);
      __syncthreads();
      for (int e = tid; e < 32 * 32; e += 256) {
        const int a = e & 31, c = e >> 5;
        L11[a][c] = (a < pw && c < pw && a >= c) ? L[(size_t)(p0 + c) * b + p0 + a] : 0.0;
      }
      if (tid < 32) dinv[tid] = tid < pw ? 1.0 / L[(size_t)(p0 + tid) * b + p0 + tid] : 0.0;
      __syncthreads();
      // diagonal block solve, one thread per column
      if (tid < rq) {
        double* vc = Vt + (size_t)(q0 + tid) * b + p0;
        double x[32];
#pragma unroll
        for (int a = 0; a < 32; ++a) x[a] = (a < pw) ? vc[a] : 0.0;
#pragma unroll
        for (int a = 0; a < 32; ++a) {
          if (a < pw) {
            double s = x[a];
#pragma unroll
            for (int c = 0; c < a; ++c) s -= L11[a][c] * x[c];
            x[a] = s * dinv[a];
          }
        }
#pragma unroll
        for (int a = 0; a < 32; ++a)
          if (a < pw) { vc[a] = x[a]; Xp[a][tid] = x[a]; }
      }
      __syncthreads();
      // update rows below: V[row, q] -= sum_c L[row, p0 + c] X[c, q]
      for (int row = p0 + pw + tid; row < bk; row += 256) {
        double l[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) l[c] = (c < pw) ? L[(size_t)(p0 + c) * b + row] : 0.0;
        // eight columns of V at a time: their current values are loaded together, then the dots
        for (int q1 = 0; q1 < rq; q1 += 8) {
          double old[8], sv[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            old[u] = q1 + u < rq ? Vt[(size_t)(q0 + q1 + u) * b + row] : 0.0;
            sv[u] = 0.0;
          }
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const double lc = l[c];
#pragma unroll
            for (int u = 0; u < 8; ++u) sv[u] = fma(lc, Xp[c][min(q1 + u, 63)], sv[u]);
          }
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (q1 + u < rq) Vt[(size_t)(q0 + q1 + u) * b + row] = old[u] - sv[u];
        }
      }
    }
  }
  __syncthreads();
  if (round_store) {  // storage rule 'mixed': the factor tile rounded under the full budget (17:183-184)
    __shared__ double rred[40];
    const int bits = cta_round_pair(Ut, Vt, bi, bk, r, b, thr_abs, rred, rmode == kRankReplay ? blog_trsm[t] : 0);
    if (tid == 0) {
      prec[t] = bits;
      if (rmode == kRankRecord) blog_trsm[t] = bits;
    }
  }
  // W = V^T V (r x r) and t = V^T z_k
  const double* zk = z + (size_t)k * b;
  double* W = Wd + (size_t)t * cap * cap;
  for (int e = warp; e < r * r + r; e += 8) {
    double s = 0.0;
    if (e < r * r) {
      const int p = e % r, q = e / r;
      if (p <= q) {
        const double* vp = Vt + (size_t)p * b;
        const double* vq = Vt + (size_t)q * b;
        for (int a = lane; a < bk; a += 32) s += vp[a] * vq[a];
        s = warp_sum(s);
        if (lane == 0) { W[(size_t)q * cap + p] = s; W[(size_t)p * cap + q] = s; }
      }
    } else {
      const int p = e - r * r;
      const double* vp = Vt + (size_t)p * b;
      for (int a = lane; a < bk; a += 32) s += vp[a] * zk[a];
      s = warp_sum(s);
      if (lane == 0 && p < 64) zt[p] = s;
    }
  }
  __syncthreads();
  // Y_ik = U_ik W_ik, the factor of the deferred diagonal update of tile i
  double* Yt = Y + (size_t)t * b * cap;
  for (int a = tid; a < bi; a += 256)
    for (int q1 = 0; q1 < r; q1 += 8) {  // eight output columns per pass over the row of U
      double sv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) sv[u] = 0.0;
      for (int p = 0; p < r; ++p) {
        const double up = Ut[(size_t)p * b + a];
#pragma unroll
        for (int u = 0; u < 8; ++u) sv[u] = fma(up, W[(size_t)min(q1 + u, r - 1) * cap + p], sv[u]);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (q1 + u < r) Yt[(size_t)(q1 + u) * b + a] = sv[u];
    }
  double* ri = rhs + (size_t)i * b;
  if (r <= 64) {
    for (int a = tid; a < bi; a += 256) {
      double s = 0.0;
      for (int q = 0; q < r; ++q) s = fma(Ut[(size_t)q * b + a], zt[q], s);
      ri[a] -= s;
    }
  } else {
    // wider ranks: recompute the projections column by column (rare)
    for (int a = tid; a < bi; a += 256) {
      double s = 0.0;
      for (int q = 0; q < r; ++q) {
        double tq = 0.0;
        const double* vq = Vt + (size_t)q * b;
        for (int u = 0; u < bk; ++u) tq += vq[u] * zk[u];
        s = fma(Ut[(size_t)q * b + a], tq, s);
      }
      ri[a] -= s;
    }
  }
}

// ----------------------------------------------------------------------------------------
// Recompression of the trailing tiles at step k.  Persistent grid; each CTA owns one slot of
// global scratch (L2-resident working arrays).
struct RcScratch {
  double *W, *Cc, *Dd, *X, *Y, *Ru, *Rv, *M, *Vs, *G, *Hh, *Uo, *Vo;
};

__device__ RcScratch rc_slot(double* base, int b, int cap) {
  const size_t c2 = (size_t)cap * cap, s2 = (size_t)4 * cap * cap, bc = (size_t)b * cap;
  RcScratch s;
  double* p = base;
  s.W = p; p += c2;
  s.Cc = p; p += c2;
  s.Dd = p; p += c2;
  s.X = p; p += bc;
  s.Y = p; p += bc;
  s.Ru = p; p += s2;
  s.Rv = p; p += s2;
  s.M = p; p += s2;
  s.Vs = p; p += s2;
  s.G = p; p += 2 * c2;
  s.Hh = p; p += c2;
  s.Uo = p; p += bc;
  s.Vo = p; p += bc;
  return s;
}

size_t rc_slot_doubles(int b, int cap) {
  const size_t c2 = (size_t)cap * cap, bc = (size_t)b * cap;
  return 3 * c2 + 2 * bc + 4 * 4 * c2 + 2 * c2 + c2 + 2 * bc;
}

// C (p x q, ld p) = A^T B with A (m x p, lda), B (m x q, ldb): one warp per entry.
__device__ void cta_atb(const double* A, int lda, const double* B, int ldb, int m, int p, int q, double* C,
                        int ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int e = warp; e < p * q; e += nwarp) {
    const int u = e % p, v = e / p;
    const double* a = A + (size_t)u * lda;
    const double* bb = B + (size_t)v * ldb;
    double s = 0.0;
    for (int t = lane; t < m; t += 32) s += a[t] * bb[t];
    s = warp_sum(s);
    if (lane == 0) C[(size_t)v * ldc + u] = s;
  }
}

// One task of cta_atb4 (task e of p * ceil(q / 4): row u of C, four consecutive columns), by one warp.
__device__ __forceinline__ void atb4_task(const double* A, int lda, const double* B, int ldb, int m, int p, int q,
                                          double* C, int ldc, const double* scale, int e) {
  const int lane = threadIdx.x & 31;
  {
    const int u = e % p, v0 = (e / p) * 4;
    const double* a = A + (size_t)u * lda;
    const double* b0 = B + (size_t)v0 * ldb;
    const double* b1 = B + (size_t)min(v0 + 1, q - 1) * ldb;
    const double* b2 = B + (size_t)min(v0 + 2, q - 1) * ldb;
    const double* b3 = B + (size_t)min(v0 + 3, q - 1) * ldb;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int t = lane; t < m; t += 32) {
      const double x = a[t];
      s0 += x * b0[t];
      s1 += x * b1[t];
      s2 += x * b2[t];
      s3 += x * b3[t];
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    s3 = warp_sum(s3);
    if (lane == 0) {
      const double sc = scale ? scale[u] : 1.0;
      C[(size_t)v0 * ldc + u] = scale ? s0 * sc : s0;
      if (v0 + 1 < q) C[(size_t)(v0 + 1) * ldc + u] = scale ? s1 * sc : s1;
      if (v0 + 2 < q) C[(size_t)(v0 + 2) * ldc + u] = scale ? s2 * sc : s2;
      if (v0 + 3 < q) C[(size_t)(v0 + 3) * ldc + u] = scale ? s3 * sc : s3;
    }
  }
}

// C[v][u] = (sum_t A[u][t] B[v][t]) (times scale[u] when scale is given) for u < p, v < q, column v
// of C at C + v ldc.  One warp per (u, four consecutive v), so A's column is read once for four
// dots; every entry is summed as in cta_atb (lane t = lane, lane + 32, ..., then the butterfly),
// so the results are cta_atb's bit for bit.
__device__ void cta_atb4(const double* A, int lda, const double* B, int ldb, int m, int p, int q, double* C,
                         int ldc, const double* scale) {
  const int warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int ntask = p * ((q + 3) >> 2);
  for (int e = warp; e < ntask; e += nwarp) atb4_task(A, lda, B, ldb, m, p, q, C, ldc, scale, e);
}

// General recompression of one trailing pair, the reference's recompress as written
// (codes/17_tlr_cholesky_pilot.py:119-133): Householder QR of A = [U_ij, -U_ik W] and
// B = [V_ij, U_jk] (no orthogonality assumed), SVD of the core R_u R_v^T by one-sided Jacobi on
// its transpose, the rule's rank, U' = Q_u U_w s, V' = Q_v V_w.  The storage rule 'mixed' uses it:
// its rounded factors are no longer orthogonal, which the structured projection needs.  The new
// pair overwrites the tile (i, j); with round_store it is then rounded under the budget left after
// truncation (17:203-204).  Returns the new rank, or -1 after setting an error status.
__device__ int rc_general_pair(int bi, int bj, int b, int cap, int r1, int ri, int rj, const double* Uik,
                               const double* Ujk, const double* W, double* Uw, double* Vw, RcScratch& S,
                               double* sig, int* perm, int* iflag, double* red, int* rsel, int rule_fixed,
                               double thr_rel, double thr_abs, int round_store, int* rlog_pp, int* blog_pp,
                               int rmode, int* status) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int s = r1 + rj, ls = 2 * cap;
  const int ku = min(bi, s), kv = min(bj, s);
  double* A = S.X;   // b x 2 cap (X and Y are contiguous)
  double* B = S.Uo;  // b x 2 cap (Uo and Vo are contiguous)
  for (int q = 0; q < r1; ++q) {
    for (int a = tid; a < bi; a += nt) A[(size_t)q * b + a] = Uw[(size_t)q * b + a];
    for (int a = tid; a < bj; a += nt) B[(size_t)q * b + a] = Vw[(size_t)q * b + a];
  }
  for (int q = 0; q < rj; ++q) {
    for (int a = tid; a < bi; a += nt) {
      double acc = 0.0;
      for (int p = 0; p < ri; ++p) acc = fma(Uik[(size_t)p * b + a], W[(size_t)q * cap + p], acc);
      A[(size_t)(r1 + q) * b + a] = -acc;
    }
    for (int a = tid; a < bj; a += nt) B[(size_t)(r1 + q) * b + a] = Ujk[(size_t)q * b + a];
  }
  __syncthreads();
  // A = Q_u R_u, B = Q_v R_v (R upper trapezoidal ku x s / kv x s, Q explicit bi x ku / bj x kv)
  cta_geqr2(A, b, bi, s, sig, red);
  cta_copy_r(A, b, ku, s, S.Ru, ls);
  cta_org2r(A, b, bi, ku, sig);
  cta_geqr2(B, b, bj, s, sig, red);
  cta_copy_r(B, b, kv, s, S.Rv, ls);
  cta_org2r(B, b, bj, kv, sig);
  // Z = (R_u R_v^T)^T (kv x ku): Z[c][a] = sum_t R_u[a][t] R_v[c][t], t >= max(a, c)
  for (int e = tid; e < ku * kv; e += nt) {
    const int c = e % kv, a = e / kv;
    double acc = 0.0;
    for (int t = max(a, c); t < s; ++t) acc = fma(S.Ru[(size_t)t * ls + a], S.Rv[(size_t)t * ls + c], acc);
    S.M[(size_t)a * ls + c] = acc;
  }
  __syncthreads();
  // Z J = Z' (orthogonal columns): core = J Z'^T, left singular vectors J, right Z' / sigma
  cta_jacobi_svd(S.M, ls, kv, ku, S.Vs, ls, sig, perm, iflag, 40, 1e-28);
  if (tid == 0) {
    double srt[256];
    double fro2 = 0.0;
    for (int q = 0; q < ku; ++q) srt[q] = sig[perm[q]];
    for (int q = ku - 1; q >= 0; --q) fro2 += srt[q] * srt[q];
    const double thr = rule_fixed ? thr_rel * sqrt(fro2) : thr_abs;
    int r = select_rank(srt, ku, 0.0, thr, nullptr);
    if (r < 0) r = ku;
    if (rmode == kRankReplay) r = min(*rlog_pp, ku);
    else if (rmode == kRankRecord) *rlog_pp = r;
    double tail2 = 0.0;
    for (int q = ku - 1; q >= r; --q) tail2 += srt[q] * srt[q];
    if (r > cap) {
      atomicCAS(status, 0, -2);
      r = -1;
    }
    rsel[0] = r;
    reinterpret_cast<double*>(rsel + 2)[0] = sqrt(tail2);
  }
  __syncthreads();
  const int rn = rsel[0];
  const double tail = reinterpret_cast<double*>(rsel + 2)[0];
  if (rn < 0) return -1;
  // U' = Q_u (J[:, perm c] sigma), V' = Q_v (Z'[:, perm c] / sigma): over the tile's own slot
  for (int c = 0; c < rn; ++c) {
    const int pc = perm[c];
    const double sg = sig[pc], inv = sg > 0.0 ? 1.0 / sg : 0.0;
    const double* jc = S.Vs + (size_t)pc * ls;
    const double* zc = S.M + (size_t)pc * ls;
    for (int a = tid; a < bi; a += nt) {
      double acc = 0.0;
      for (int q = 0; q < ku; ++q) acc = fma(A[(size_t)q * b + a], jc[q], acc);
      Uw[(size_t)c * b + a] = acc * sg;
    }
    for (int a = tid; a < bj; a += nt) {
      double acc = 0.0;
      for (int q = 0; q < kv; ++q) acc = fma(B[(size_t)q * b + a], zc[q], acc);
      Vw[(size_t)c * b + a] = acc * inv;
    }
  }
  __syncthreads();
  if (round_store) {
    const int bits = cta_round_pair(Uw, Vw, bi, bj, rn, b, thr_abs - tail, red, rmode == kRankReplay ? *blog_pp : 0);
    if (tid == 0 && rmode == kRankRecord) *blog_pp = bits;
  }
  return rn;
}

// The mixed path uses this kernel as it stands.  Three ways of making it cheaper there were measured
// on the N = 50,000 bench workload and withdrawn: one Gram-Schmidt pass without re-orthogonalising
// Q3 (5.53 against 5.09 evals/s, but 0.024 nats and 2e-3 of the gradient from FP64, over the
// budget), a core Jacobi that stops at |cos| <= 1e-10 (no faster, 0.0079 nats, over budget on three
// N = 20,000 sweep fields), 128-thread CTAs at 6 or 8 per SM (recompression 279 / 318 ms
// against 175 ms per evaluation), and 256-thread CTAs at 5 or 6 per SM (48 / 40 registers, which
// spill: 237 / 272 ms against 188 ms in the same run, batched mixed 4.30 / 4.05 against 4.83
// evals/s).
constexpr int kRcSmemS = 32;  // cores with s <= 32 are solved in shared memory
#ifndef TLR_RC_THREADS
#define TLR_RC_THREADS 256
#endif
constexpr int kRcT = TLR_RC_THREADS;  // threads per pair
constexpr int kRcW = kRcT / 32;
#ifndef TLR_RC_BLOCKS
#define TLR_RC_BLOCKS 3
#endif
#ifndef TLR_RC_CHUNK
#define TLR_RC_CHUNK 8
#endif
constexpr int kRcCW = TLR_RC_CHUNK;  // output columns per pass over a row in the row loops
constexpr int kRcMinBlocks = TLR_RC_BLOCKS;  // resident CTAs per SM (the register cap follows)

int rc_blocks_per_sm() { return kRcMinBlocks; }

// Trailing pairs held by the first m of a rank's rows ii0, ii0 + w, ... (row ii holds ii pairs).
__host__ __device__ inline long rc_pairs_before(long m, long ii0, long w) { return m * ii0 + w * m * (m - 1) / 2; }

__global__ void __launch_bounds__(kRcT, kRcMinBlocks) k_recompress(int n, int b, int k, int nB, double* TLR_RESTRICT U,
                                                   double* TLR_RESTRICT V, int* TLR_RESTRICT rank, int cap,
                                                   double* TLR_RESTRICT scratch, size_t slot_doubles,
                                                   int* TLR_RESTRICT next_pair, int* TLR_RESTRICT rlog,
                                                   int* TLR_RESTRICT blog, int prank, int pworld,
                                                   int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const EvalParams& prm = *eval_params(status);
  const int rule_fixed = prm.rule_fixed, rmode = prm.rmode, round_store = prm.round_store;
  const int general = round_store;  // rounded factors are not orthogonal: the general recompression
  const double thr_rel = prm.thr_rel, thr_abs = prm.thr_abs;
  const int mB = nB - k - 1;  // trailing tiles
  // the pairs (i, j), k < j < i, of this rank's trailing rows ii = ii0 + m pworld (i = k + 1 + ii,
  // i % pworld == prank; every row when pworld = 1): row ii holds ii pairs, so rows 0..m-1 of the
  // rank hold C(m) = m ii0 + pworld m (m - 1) / 2
  const long ii0 = ((prank - (k + 1)) % pworld + pworld) % pworld;
  const long mown = ii0 < mB ? (mB - 1 - ii0) / pworld + 1 : 0;
  const long npairs = rc_pairs_before(mown, ii0, pworld);
  RcScratch S = rc_slot(scratch + (size_t)blockIdx.x * slot_doubles, b, cap);
  extern __shared__ double rc_smem[];
  double* Msm = rc_smem;                            // kRcSmemS^2
  double* Vsm = rc_smem + kRcSmemS * kRcSmemS;      // kRcSmemS^2
  double* Zsm = rc_smem + 2 * kRcSmemS * kRcSmemS;  // kRcSmemS^2
  __shared__ double red[40];
  __shared__ double n1[128];
  __shared__ double ninv[128];
  __shared__ double nvv[128];
  __shared__ double nvinv[128];
  __shared__ double sig[256];
  __shared__ int perm[256];
  __shared__ int iflag[2];
  __shared__ int rsel;
  __shared__ __align__(8) int gsel[4];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ls = 2 * cap;
  if (blockIdx.x == 0 && tid == 0) {  // the panel column k is read once per step
    double by = 0.0;
    for (int i = k + 1; i < nB; ++i) by += 8.0 * 2.0 * b * rank[tidx(i, k)];
    add_work(status, 10, 0.0, by);
  }
  // pairs are handed out dynamically: each CTA starts on pair blockIdx.x and then takes the next
  // unclaimed one (*next_pair counts the claims past the grid; zero at launch), so CTAs that drew
  // low-rank pairs take more of them
  __shared__ long q_next;
  auto claim = [&]() -> long {
    __syncthreads();
    if (threadIdx.x == 0) q_next = (long)gridDim.x + atomicAdd(next_pair, 1);
    __syncthreads();
    return q_next;
  };
  for (long qq = blockIdx.x; qq < npairs; qq = claim()) {
    // decode qq -> (row m of the rank, jj), then pp = the pair's index among all trailing pairs
    const double hb = (double)ii0 - 0.5 * pworld;
    long m = (long)((-hb + sqrt(hb * hb + 2.0 * pworld * (double)qq)) / pworld);
    while (m > 0 && rc_pairs_before(m, ii0, pworld) > qq) --m;
    while (rc_pairs_before(m + 1, ii0, pworld) <= qq) ++m;
    const int ii = (int)(ii0 + m * pworld);
    const int jj = (int)(qq - rc_pairs_before(m, ii0, pworld));
    const long pp = (long)ii * (ii - 1) / 2 + jj;
    const int i = k + 1 + ii, j = k + 1 + jj;
    const int tij = tidx(i, j), tik = tidx(i, k), tjk = tidx(j, k);
    const int r1 = rank[tij], ri = rank[tik], rj = rank[tjk];
    if (ri == 0 || rj == 0) continue;
    const int bi = min(b, n - i * b), bj = min(b, n - j * b), bk = min(b, n - k * b);
    const double* Uij = U + (size_t)tij * b * cap;
    const double* Vij = V + (size_t)tij * b * cap;
    const double* Uik = U + (size_t)tik * b * cap;
    const double* Vik = V + (size_t)tik * b * cap;
    const double* Ujk = U + (size_t)tjk * b * cap;
    const double* Vjk = V + (size_t)tjk * b * cap;
    const int s = r1 + rj;
    const bool core_in_smem = s <= kRcSmemS;
    double* Mc = core_in_smem ? Msm : S.M;
    double* Vc = core_in_smem ? Vsm : S.Vs;
    double* Zc = core_in_smem ? Zsm : S.Ru;  // R_u is no longer needed once M is formed
    const int lc = core_in_smem ? kRcSmemS : ls;
    __syncthreads();
    // W = V_ik^T V_jk (ri x rj); column norms of U_ij
    // W's dot tasks and the column norms share one round-robin over the warps
    const int nW = ri * ((rj + 3) >> 2);
    for (int e = warp; e < nW + r1; e += kRcW) {
      if (e < nW) {
        atb4_task(Vik, b, Vjk, b, bk, ri, rj, S.W, cap, nullptr, e);
        continue;
      }
      const int c = e - nW;
      const double* u = Uij + (size_t)c * b;
      const double* v = Vij + (size_t)c * b;
      double a = 0.0, av = 0.0;
      for (int t = lane; t < bi; t += 32) a += u[t] * u[t];
      for (int t = lane; t < bj; t += 32) av += v[t] * v[t];
      a = warp_sum(a);
      av = warp_sum(av);
      if (lane == 0) {
        n1[c] = sqrt(a);
        ninv[c] = a > 0.0 ? 1.0 / sqrt(a) : 0.0;
        nvv[c] = sqrt(av);
        nvinv[c] = av > 0.0 ? 1.0 / sqrt(av) : 0.0;
      }
    }
    __syncthreads();
    if (general) {  // storage rule 'mixed': the reference's recompression as written
      const int rn = rc_general_pair(bi, bj, b, cap, r1, ri, rj, Uik, Ujk, S.W, U + (size_t)tij * b * cap,
                                     V + (size_t)tij * b * cap, S, sig, perm, iflag, red, gsel, rule_fixed,
                                     thr_rel, thr_abs, round_store, rlog + pp, blog + pp, rmode, status);
      if (rn < 0) return;
      if (tid == 0) {
        rank[tij] = rn;
        add_work(status, 10, 4.0 * b * ri * rj + 16.0 * b * s * s + 4.0 * b * s * rn,
                 8.0 * ((double)(bi + bj) * r1 + (double)(bi + bj) * rn));
      }
      __syncthreads();
      continue;
    }
    // X = -U_ik W (bi x rj), kRcCW columns per pass over a row of U_ik
    for (int a = tid; a < bi; a += kRcT)
      for (int q0 = 0; q0 < rj; q0 += kRcCW) {
        double acc[kRcCW] = {};
        for (int p = 0; p < ri; ++p) {
          const double x = Uik[(size_t)p * b + a];
#pragma unroll
          for (int w = 0; w < kRcCW; ++w) acc[w] = fma(x, S.W[(size_t)min(q0 + w, rj - 1) * cap + p], acc[w]);
        }
#pragma unroll
        for (int w = 0; w < kRcCW; ++w)
          if (q0 + w < rj) S.X[(size_t)(q0 + w) * b + a] = -acc[w];
      }
    __syncthreads();
    // block Gram-Schmidt twice against Q1 = U_ij diag(1/n1): C = Q1^T X, X -= Q1 C
    for (int pass = 0; pass < 2; ++pass) {
      if (r1 > 0) {
        cta_atb4(Uij, b, S.X, b, bi, r1, rj, S.G, cap, ninv);  // C increment
        __syncthreads();
        for (int a = tid; a < bi; a += kRcT)
          for (int v0 = 0; v0 < rj; v0 += kRcCW) {
            double acc[kRcCW] = {};
            for (int u = 0; u < r1; ++u) {
              const double x = Uij[(size_t)u * b + a] * ninv[u];
#pragma unroll
              for (int w = 0; w < kRcCW; ++w) acc[w] = fma(x, S.G[(size_t)min(v0 + w, rj - 1) * cap + u], acc[w]);
            }
#pragma unroll
            for (int w = 0; w < kRcCW; ++w)
              if (v0 + w < rj) S.X[(size_t)(v0 + w) * b + a] -= acc[w];
          }
        for (int e = tid; e < r1 * rj; e += kRcT) {
          const int u = e % r1, v = e / r1;
          const double inc = S.G[(size_t)v * cap + u];
          S.Cc[(size_t)v * cap + u] = pass == 0 ? inc : S.Cc[(size_t)v * cap + u] + inc;
        }
      }
      __syncthreads();
    }
    // R2 from Householder QR of the projected X (bi x rj); its reflectors are not needed
    cta_geqr2_r(S.X, b, bi, rj, red);
    // V side: D = V_ij^T U_jk, Y = U_jk - V_ij D (twice; the first pass reads U_jk itself)
    if (r1 == 0) {
      for (int v = 0; v < rj; ++v)
        for (int a = tid; a < bj; a += kRcT) S.Y[(size_t)v * b + a] = Ujk[(size_t)v * b + a];
      __syncthreads();
    }
    for (int pass = 0; pass < 2; ++pass) {
      if (r1 > 0) {
        const double* Yin = pass == 0 ? Ujk : S.Y;
        cta_atb4(Vij, b, Yin, b, bj, r1, rj, S.G, cap, nvinv);
        __syncthreads();
        for (int a = tid; a < bj; a += kRcT)
          for (int v0 = 0; v0 < rj; v0 += kRcCW) {
            double acc[kRcCW] = {};
            for (int u = 0; u < r1; ++u) {
              const double x = Vij[(size_t)u * b + a] * nvinv[u];
#pragma unroll
              for (int w = 0; w < kRcCW; ++w) acc[w] = fma(x, S.G[(size_t)min(v0 + w, rj - 1) * cap + u], acc[w]);
            }
#pragma unroll
            for (int w = 0; w < kRcCW; ++w)
              if (v0 + w < rj) S.Y[(size_t)(v0 + w) * b + a] = Yin[(size_t)(v0 + w) * b + a] - acc[w];
          }
        for (int e = tid; e < r1 * rj; e += kRcT) {
          const int u = e % r1, v = e / r1;
          const double inc = S.G[(size_t)v * cap + u];
          S.Dd[(size_t)v * cap + u] = pass == 0 ? inc : S.Dd[(size_t)v * cap + u] + inc;
        }
      }
      __syncthreads();
    }
    // R_u = [[diag(n1), C], [0, R2]] (s x s, ld ls)
    for (int e = tid; e < s * s; e += kRcT) {  // entry (a, c); every small loop below is flat too
        const int a = e % s, c = e / s;
        double vu = 0.0;
        if (a < r1) vu = (c < r1) ? (a == c ? n1[a] : 0.0) : S.Cc[(size_t)(c - r1) * cap + a];
        else if (c >= r1 && a <= c && a - r1 < bi) vu = S.X[(size_t)(c - r1) * b + (a - r1)];
        S.Ru[(size_t)c * ls + a] = vu;
      }
    __syncthreads();
    double* tau3 = sig + 128;
    cta_geqr2(S.Y, b, bj, rj, tau3, red);
    // R_v = [[I, D], [0, R3]]
    for (int e = tid; e < s * s; e += kRcT) {
        const int a = e % s, c = e / s;
        double vv = 0.0;
        if (a < r1) vv = (c < r1) ? (a == c ? nvv[a] : 0.0) : S.Dd[(size_t)(c - r1) * cap + a];
        else if (c >= r1 && a <= c && a - r1 < bj) vv = S.Y[(size_t)(c - r1) * b + (a - r1)];
        S.Rv[(size_t)c * ls + a] = vv;
      }
    __syncthreads();
    cta_org2r(S.Y, b, bj, rj, tau3);
    if (rj > bj) {  // a ragged tile shorter than the rank: the extra basis columns are zero
      for (int v = bj; v < rj; ++v)
        for (int a = tid; a < bj; a += kRcT) S.Y[(size_t)v * b + a] = 0.0;
      __syncthreads();
    }
    // re-orthogonalise Q3 against the normalised V_ij once
    if (r1 > 0) {
      cta_atb4(Vij, b, S.Y, b, bj, r1, rj, S.G, cap, nullptr);
      __syncthreads();
      for (int a = tid; a < bj; a += kRcT)
        for (int v0 = 0; v0 < rj; v0 += kRcCW) {
          double acc[kRcCW] = {};
          for (int u = 0; u < r1; ++u) {
            const double x = Vij[(size_t)u * b + a] * nvinv[u];
#pragma unroll
            for (int w = 0; w < kRcCW; ++w)
              acc[w] = fma(x, S.G[(size_t)min(v0 + w, rj - 1) * cap + u] * nvinv[u], acc[w]);
          }
#pragma unroll
          for (int w = 0; w < kRcCW; ++w)
            if (v0 + w < rj) S.Y[(size_t)(v0 + w) * b + a] -= acc[w];
        }
      __syncthreads();
    }
    // core M = R_u R_v^T (s x s); both factors are upper triangular
    for (int e = tid; e < s * s; e += kRcT) {
        const int a = e % s, c = e / s;
        double acc = 0.0;
        const int t0 = a > c ? a : c;
        for (int t = t0; t < s; ++t) acc = fma(S.Ru[(size_t)t * ls + a], S.Rv[(size_t)t * ls + c], acc);
        Mc[(size_t)c * lc + a] = acc;
      }
    __syncthreads();
    // SVD of the core: Householder QR M = Q_M R_M, then one-sided Jacobi on R_M^T (R_M^T W = Z,
    // orthogonal columns, sigma = column norms), so M = Q_M W Z^T and the right singular vectors
    // are the normalised columns of Z.  The QR grades the columns, so the Jacobi needs 3-5 sweeps
    // instead of 6-16 on M itself.
    cta_geqr2_r(Mc, lc, s, s, red);
    for (int e = tid; e < s * s; e += kRcT) {
      const int a = e % s, c = e / s;
      Zc[(size_t)c * lc + a] = (a >= c) ? Mc[(size_t)a * lc + c] : 0.0;
    }
    __syncthreads();
    // columns below 1e-14 of the largest singular value (the projections' rounding noise) are not
    // rotated: their relative orthogonality test would otherwise run to the sweep limit
    cta_jacobi_svd(Zc, lc, s, s, nullptr, lc, sig, perm, iflag, 40, 1e-28);  // only Z is used
    // Vc <- normalised Z (right singular vectors of M); the rotation matrix is not formed
    for (int c = warp; c < s; c += kRcW) {
      const double inv = sig[c] > 0.0 ? 1.0 / sig[c] : 0.0;
      for (int a = lane; a < s; a += 32) Vc[(size_t)c * lc + a] = Zc[(size_t)c * lc + a] * inv;
    }
    __syncthreads();
    if (tid == 0) {
      double srt[256];
      double fro2 = 0.0;
      for (int q = 0; q < s; ++q) srt[q] = sig[perm[q]];
      for (int q = s - 1; q >= 0; --q) fro2 += srt[q] * srt[q];
      const double thr = rule_fixed ? thr_rel * sqrt(fro2) : thr_abs;
      int r = select_rank(srt, s, 0.0, thr, nullptr);
      if (r < 0) r = s;
      if (rmode == kRankReplay) r = min(rlog[pp], s);  // frozen: the rank recorded at another theta
      else if (rmode == kRankRecord) rlog[pp] = r;
      if (r > cap) {
        atomicCAS(status, 0, -2);
        r = -1;
      }
      rsel = r;
    }
    __syncthreads();
    const int rn = rsel;
    if (rn < 0) return;
    if (tid == 0)  // 4 b r_ik r_jk + 8 b s^2 + 4 b s r' flops; old and new pair read / written
      add_work(status, 10, 4.0 * b * ri * rj + 8.0 * b * s * s + 4.0 * b * s * rn,
               8.0 * ((double)(bi + bj) * r1 + (double)(bi + bj) * rn));
    // G = R_v^T Vs_r (s x rn), H = W G_bottom (ri x rn)
    for (int e = tid; e < s * rn; e += kRcT) {
        const int t = e % s, c = e / s;
        const double* vc = Vc + (size_t)perm[c] * lc;
        double acc = 0.0;
        for (int a = 0; a <= t; ++a) acc = fma(S.Rv[(size_t)t * ls + a], vc[a], acc);
        S.G[(size_t)c * ls + t] = acc;
      }
    __syncthreads();
    for (int e = tid; e < ri * rn; e += kRcT) {
      const int p = e % ri, c = e / ri;
      double acc = 0.0;
      for (int q = 0; q < rj; ++q) acc = fma(S.W[(size_t)q * cap + p], S.G[(size_t)c * ls + r1 + q], acc);
      S.Hh[(size_t)c * cap + p] = acc;
    }
    __syncthreads();
    // U' = U_ij G_top - U_ik H ; V' = V_ij Vs_top + Q3 Vs_bottom, kRcCW columns per pass over a row.
    // With rn <= kRcCW one pass makes a row's every output after reading all its inputs (each thread
    // reads and writes its own rows only), so the new pair goes straight over the old one.
    double* Uw = U + (size_t)tij * b * cap;
    double* Vw = V + (size_t)tij * b * cap;
    const bool direct = rn <= kRcCW;
    double* Uout = direct ? Uw : S.Uo;
    double* Vout = direct ? Vw : S.Vo;
    for (int a = tid; a < bi; a += kRcT)
      for (int c0 = 0; c0 < rn; c0 += kRcCW) {
        double acc[kRcCW] = {};
        for (int t = 0; t < r1; ++t) {
          const double x = Uij[(size_t)t * b + a];
#pragma unroll
          for (int w = 0; w < kRcCW; ++w) acc[w] = fma(x, S.G[(size_t)min(c0 + w, rn - 1) * ls + t], acc[w]);
        }
        for (int p = 0; p < ri; ++p) {
          const double x = -Uik[(size_t)p * b + a];
#pragma unroll
          for (int w = 0; w < kRcCW; ++w) acc[w] = fma(x, S.Hh[(size_t)min(c0 + w, rn - 1) * cap + p], acc[w]);
        }
#pragma unroll
        for (int w = 0; w < kRcCW; ++w)
          if (c0 + w < rn) Uout[(size_t)(c0 + w) * b + a] = acc[w];
      }
    for (int a = tid; a < bj; a += kRcT)
      for (int c0 = 0; c0 < rn; c0 += kRcCW) {
        int vo[kRcCW];  // offsets of the chunk's right singular vectors in Vc
#pragma unroll
        for (int w = 0; w < kRcCW; ++w) vo[w] = perm[min(c0 + w, rn - 1)] * lc;
        double acc[kRcCW] = {};
        for (int t = 0; t < r1; ++t) {
          const double x = Vij[(size_t)t * b + a] * nvinv[t];
#pragma unroll
          for (int w = 0; w < kRcCW; ++w) acc[w] = fma(x, Vc[vo[w] + t], acc[w]);
        }
        for (int t = 0; t < rj; ++t) {
          const double x = S.Y[(size_t)t * b + a];
#pragma unroll
          for (int w = 0; w < kRcCW; ++w) acc[w] = fma(x, Vc[vo[w] + r1 + t], acc[w]);
        }
#pragma unroll
        for (int w = 0; w < kRcCW; ++w)
          if (c0 + w < rn) Vout[(size_t)(c0 + w) * b + a] = acc[w];
      }
    if (!direct) {
      __syncthreads();
      for (int c = 0; c < rn; ++c) {
        for (int a = tid; a < bi; a += kRcT) Uw[(size_t)c * b + a] = S.Uo[(size_t)c * b + a];
        for (int a = tid; a < bj; a += kRcT) Vw[(size_t)c * b + a] = S.Vo[(size_t)c * b + a];
      }
    }
    if (tid == 0) rank[tij] = rn;
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------------------
__global__ void k_finish(int nB, int n, const double* ldpart, const double* qpart, double* out,
                         const int* status) {
  if (threadIdx.x != 0) return;
  if (*status != 0) { out[0] = 0.0; out[1] = 0.0; out[2] = 0.0; return; }
  double ld = 0.0, q = 0.0;
  for (int k = 0; k < nB; ++k) { ld += ldpart[k]; q += qpart[k]; }
  const double log2pi = 1.8378770664093454836;
  out[0] = -0.5 * (q + ld + (double)n * log2pi);
  out[1] = ld;
  out[2] = q;
}

// ----------------------------------------------------------------------------------------
int launch_diag_build(const double* xy, int n, int b, int k, const double* U, const double* Y, const int* rank,
                      int cap, double* D, const int* status, cudaStream_t s) {
  const int bk = std::min(b, n - k * b);
  const int nb = (bk + 31) / 32;
  k_diag_build<<<nb * (nb + 1) / 2, 256, 0, s>>>(xy, n, b, k, U, Y, rank, cap, D, status);
  return (int)cudaGetLastError();
}

int launch_trsm(const double* D, int n, int b, int k, int nB, double* U, double* V, double* Wd, double* Y,
                const int* rank, int cap, const double* z, double* rhs, int* prec, int* blog_trsm, int prank,
                int pworld, const int* status, cudaStream_t s) {
  if (nB - k - 1 <= 0) return 0;
  k_trsm<<<nB - k - 1, 256, 0, s>>>(D, n, b, k, nB, U, V, Wd, Y, rank, cap, z, rhs, prec, blog_trsm, prank, pworld,
                                    status);
  return (int)cudaGetLastError();
}

int launch_recompress(int n, int b, int k, int nB, double* U, double* V, int* rank, int cap, double* scratch,
                      size_t slot_doubles, int nslots, int* next_pair, int* rlog_step, int* blog_step, int prank,
                      int pworld, int* status, cudaStream_t s) {
  const long mB = nB - k - 1;
  const long ii0 = ((prank - (k + 1)) % pworld + pworld) % pworld;
  const long npairs = rc_pairs_before(ii0 < mB ? (mB - 1 - ii0) / pworld + 1 : 0, ii0, pworld);
  if (npairs <= 0) return 0;
  const int grid = (int)std::min<long>(npairs, nslots);
  const size_t sm = (size_t)3 * kRcSmemS * kRcSmemS * 8;
  cudaFuncSetAttribute(k_recompress, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_recompress<<<grid, kRcT, sm, s>>>(n, b, k, nB, U, V, rank, cap, scratch, slot_doubles, next_pair, rlog_step,
                                     blog_step, prank, pworld, status);
  return (int)cudaGetLastError();
}

int launch_finish(int nB, int n, const double* ldpart, const double* qpart, double* out, const int* status,
                  cudaStream_t s) {
  k_finish<<<1, 32, 0, s>>>(nB, n, ldpart, qpart, out, status);
  return (int)cudaGetLastError();
}

}  // namespace tlr
