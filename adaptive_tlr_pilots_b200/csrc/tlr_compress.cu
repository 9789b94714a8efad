// Initial compression of the off-diagonal covariance tiles (FP64 parity path).
//
// Reference: codes/17_tlr_cholesky_pilot.py:151-166 (tile generation) and 107-116
// (truncate_svd: full SVD of every b x b tile, rank = smallest r with tail[r] <= threshold).
//
// B200 design.  A full b x b SVD per tile is O(b^3) and is where the reference spends
// 54-66% of its time.  Here each tile goes through a batched randomized range finder
// whose rank decision is exact to rounding:
//   T        generated once per chunk from the Morton-ordered coordinates (row-major, HBM);
//   Z = T^T (T P) four times, each followed by a Householder orthonormalisation (P <- Q(Z));
//   C = T P, rho^2 = ||T - C P^T||_F^2 computed element by element (no cancellation);
//   R_C from a Householder QR of C, one-sided Jacobi SVD of R_C -> sigma, W;
//   tail[r]^2 = rho^2 + sum_{t>=r} sigma_t^2 (same accumulation order as the reference);
//   the rank is accepted when r <= k - margin, so the unresolved directions lie far below
//   the threshold; otherwise the tile is redone with k doubled (16, 32, 64, 128).
// The truncated pair is U = C W_r (= Q_C U_w Sigma_r), V = P W_r, so U has orthogonal
// columns and V orthonormal columns, exactly the structure of the reference's U*s, Vt^T.
#include "tlr_device.cuh"
#include "tlr_kernels.h"

namespace tlr {

__device__ __forceinline__ double omega_entry(uint32_t tile, uint32_t row, uint32_t col) {
  // splitmix64 (Steele, Lea, Flood 2014) on (tile, row, col): a fixed, reproducible test matrix
  uint64_t x = ((uint64_t)tile << 42) ^ ((uint64_t)row << 21) ^ (uint64_t)col;
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// ----------------------------------------------------------------------------------------
// T[c] = sigma2 * matern32(dist(S_i, S_j)), row-major with leading dimension b.
__global__ void k_gen_offdiag(const double* TLR_RESTRICT xy, int n, int b, int tile_base,
                              const int* TLR_RESTRICT ti, const int* TLR_RESTRICT tj, double* TLR_RESTRICT T,
                              const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const EvalParams& prm = *eval_params(status);
  const double sigma2 = prm.sigma2, inv_range = prm.inv_range;
  const int nu5 = prm.nu5;
  const int c = blockIdx.y;
  const int t = tile_at(status, tile_base + c);
  const int i = ti[t], j = tj[t];
  const int i0 = i * b, j0 = j * b;
  const int bi = min(b, n - i0), bj = min(b, n - j0);
  double* Tc = T + (size_t)c * b * b;
  const int total = bi * bj;
  if (blockIdx.x == 0 && threadIdx.x == 0) add_work(status, 1, 0.0, 8.0 * total);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int a = e / bj, q = e - a * bj;
    const double2 pa = reinterpret_cast<const double2*>(xy)[i0 + a];
    const double2 pq = reinterpret_cast<const double2*>(xy)[j0 + q];
    Tc[(size_t)a * b + q] = matern_cov(pa.x, pa.y, pq.x, pq.y, sigma2, inv_range, nu5);
  }
}

// ----------------------------------------------------------------------------------------
// Strip-wise products with a 16-column block of P held in shared memory.
//   mode 0: Z[:, g] = T^T (T P[:, g])          (range-finder sketch)
//   mode 1: C[:, g] = T P[:, g]                 (projection)
// P is Omega (generated) when omega != 0.  One CTA of 256 threads per (tile, column group).
template <int H, int ZR>
__global__ void __launch_bounds__(256) k_sketch(const double* TLR_RESTRICT T, int n, int b, int kcols,
                                               int tile_base, const int* TLR_RESTRICT ti,
                                               const int* TLR_RESTRICT tj, const int* TLR_RESTRICT need,
                                               const double* TLR_RESTRICT P, double* TLR_RESTRICT out,
                                               int ldp, int omega, int mode, const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const int c = blockIdx.x, g = blockIdx.y;
  if (!need[c]) return;
  const int t = tile_at(status, tile_base + c);
  const int bi = min(b, n - ti[t] * b), bj = min(b, n - tj[t] * b);
  if (threadIdx.x == 0)
    add_work(status, mode == 0 ? 2 : 4, (mode == 0 ? 4.0 : 2.0) * bi * bj * 16,
             8.0 * ((double)bi * bj + (omega ? 0.0 : bj * 16.0) + (mode == 0 ? bj : bi) * 16.0));
  extern __shared__ double smem[];
  double* Ps = smem;                       // [bj][16]
  double* Ts = Ps + (size_t)b * 16;        // [H][b + 1]
  double* red = Ts + (size_t)H * (b + 1);  // [KS][H][16]
  double* Ys = red + 256 * 4;              // [H][16]
  const int ldt = b + 1;
  const double* Tc = T + (size_t)c * b * b;
  const size_t pbase = (size_t)c * b * ldp;

  for (int e = threadIdx.x; e < bj * 16; e += 256) {
    const int row = e >> 4, q = e & 15;
    Ps[e] = omega ? omega_entry((uint32_t)t, (uint32_t)row, (uint32_t)(g * 16 + q))
                  : P[pbase + (size_t)(g * 16 + q) * b + row];
  }
  constexpr int BLK = (H / 2) * 8;  // 2x2 register blocks per K slice
  constexpr int KS = 256 / BLK;     // K slices
  const int ks = threadIdx.x / BLK, loc = threadIdx.x % BLK;
  const int rp = loc >> 3, cp = loc & 7;

  double zacc[ZR][16];
#pragma unroll
  for (int m = 0; m < ZR; ++m)
#pragma unroll
    for (int q = 0; q < 16; ++q) zacc[m][q] = 0.0;

  for (int a0 = 0; a0 < bi; a0 += H) {
    const int hrows = min(H, bi - a0);
    __syncthreads();
    for (int e = threadIdx.x; e < H * bj; e += 256) {
      const int r = e / bj, q = e - r * bj;
      Ts[r * ldt + q] = (r < hrows) ? Tc[(size_t)(a0 + r) * b + q] : 0.0;
    }
    __syncthreads();
    // phase A: Y = T_s P (H x 16), 2x2 blocks, K split in KS interleaved slices
    double y00 = 0.0, y01 = 0.0, y10 = 0.0, y11 = 0.0;
    const double* t0 = Ts + (2 * rp) * ldt;
    const double* t1 = t0 + ldt;
    for (int q = ks; q < bj; q += KS) {
      const double2 pv = *reinterpret_cast<const double2*>(Ps + q * 16 + 2 * cp);
      const double a = t0[q], bb = t1[q];
      y00 = fma(a, pv.x, y00); y01 = fma(a, pv.y, y01);
      y10 = fma(bb, pv.x, y10); y11 = fma(bb, pv.y, y11);
    }
    double* rd = red + ks * (H * 16);
    rd[(2 * rp) * 16 + 2 * cp] = y00; rd[(2 * rp) * 16 + 2 * cp + 1] = y01;
    rd[(2 * rp + 1) * 16 + 2 * cp] = y10; rd[(2 * rp + 1) * 16 + 2 * cp + 1] = y11;
    __syncthreads();
    for (int e = threadIdx.x; e < H * 16; e += 256) {
      double s = 0.0;
#pragma unroll
      for (int k2 = 0; k2 < KS; ++k2) s += red[k2 * (H * 16) + e];
      Ys[e] = s;
    }
    __syncthreads();
    if (mode == 1) {
      // C rows a0.., column group g
      for (int e = threadIdx.x; e < hrows * 16; e += 256) {
        const int r = e >> 4, q = e & 15;
        out[pbase + (size_t)(g * 16 + q) * b + a0 + r] = Ys[e];
      }
      continue;
    }
    // phase B: Z += T_s^T Y
#pragma unroll
    for (int m = 0; m < ZR; ++m) {
      const int z = threadIdx.x + 256 * m;
      if (z < bj) {
        for (int r = 0; r < hrows; ++r) {
          const double a = Ts[r * ldt + z];
          const double2* yr = reinterpret_cast<const double2*>(Ys + r * 16);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const double2 yv = yr[q];
            zacc[m][2 * q] = fma(a, yv.x, zacc[m][2 * q]);
            zacc[m][2 * q + 1] = fma(a, yv.y, zacc[m][2 * q + 1]);
          }
        }
      }
    }
  }
  if (mode == 0) {
#pragma unroll
    for (int m = 0; m < ZR; ++m) {
      const int z = threadIdx.x + 256 * m;
      if (z < bj)
#pragma unroll
        for (int q = 0; q < 16; ++q) out[pbase + (size_t)(g * 16 + q) * b + z] = zacc[m][q];
    }
  }
}

// ----------------------------------------------------------------------------------------
// The same two products on the FP64 tensor cores (tiles up to 512 wide, even b).
//   One CTA of 16 warps per (tile, 16-column group); warp w owns columns [32w, 32w + 32) of T.
//   T streams through shared memory in slabs of 16 rows, double-buffered with cp.async (the
//   next slab's copy runs under this slab's products).  Per slab R:
//     phase A  Y_R = T_R P: each warp multiplies its 32-column strip by its 32 rows of P (held in
//              registers for the whole kernel) -> a 16 x 16 partial; the 16 partials are summed
//              in a fixed order (mode 1 writes that sum: the rows R of C = T P);
//     phase B  Z[strip] += T_R[:, strip]^T Y_R, accumulated in registers across slabs.
//   Every T element is read from HBM once per launch and used by both phases from shared memory.
//   MODE 0: the sketch Z = T^T T P.  MODE 1: the projection C = T P.  MODE 2 (one 16-column group,
//   k = 16): the projection and, in place of phase B, the residual of the slab on the tensor cores,
//   E_R = T_R - C_R P^T (accumulator started at T_R, operand -C_R), with rho^2 = sum E^2 and
//   ||T||^2 summed per lane in a fixed order and over the CTA in warp order into parts[c],
//   fparts[c] (one block per tile): T leaves HBM once for both.
constexpr int kSkW = 16;                 // warps per CTA
constexpr int kSkH = 16;                 // rows of T per slab
constexpr int kSkCols = 32 * kSkW;       // widest tile handled (512)
constexpr int kSkPitch = kSkCols + 4;    // slab row pitch in doubles (conflict-free fragments)
constexpr int kSkYp = 18;                // pitch of the per-warp partials
constexpr int kSkYs = 17;                // pitch of the summed Y_R

static size_t sketch_mma_smem() {
  return ((size_t)2 * kSkH * kSkPitch + (size_t)kSkW * kSkH * kSkYp + (size_t)kSkH * kSkYs) * sizeof(double);
}

template <int MODE>
__global__ void __launch_bounds__(kSkW * 32, 1)
    k_sketch_mma(const double* TLR_RESTRICT T, int n, int b, int tile_base, const int* TLR_RESTRICT ti,
                 const int* TLR_RESTRICT tj, const int* TLR_RESTRICT need, const double* TLR_RESTRICT P,
                 double* TLR_RESTRICT out, int ldp, int omega, double* TLR_RESTRICT parts,
                 double* TLR_RESTRICT fparts, const int* TLR_RESTRICT status) {
  constexpr int mode = MODE == 0 ? 0 : 1;
  if (*status != 0) return;
  const int c = blockIdx.x, grp = blockIdx.y;
  if (!need[c]) return;
  const int t = tile_at(status, tile_base + c);
  const int bi = min(b, n - ti[t] * b), bj = min(b, n - tj[t] * b);
  if (threadIdx.x == 0) {
    add_work(status, mode == 0 ? 2 : 4, (mode == 0 ? 4.0 : 2.0) * bi * bj * 16,
             8.0 * ((double)bi * bj + (omega ? 0.0 : bj * 16.0) + (mode == 0 ? bj : bi) * 16.0));
    if (MODE == 2) add_work(status, 5, 2.0 * bi * bj * 17, 0.0);
  }
  extern __shared__ __align__(16) double sk_smem[];
  double* Ts = sk_smem;                                   // [2][kSkH][kSkPitch]
  double* Yp = Ts + (size_t)2 * kSkH * kSkPitch;          // [kSkW][kSkH][kSkYp]
  double* Ys = Yp + (size_t)kSkW * kSkH * kSkYp;          // [kSkH][kSkYs]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, tg = lane & 3;
  const double* Tc = T + (size_t)c * b * b;
  const size_t pbase = (size_t)c * b * ldp;
  const int col0 = warp * 32;
  const int nslab = (bi + kSkH - 1) / kSkH;

  // slab s -> stage s & 1: kSkH rows x kSkCols columns in 16-byte pieces, zero past bi / bj
  auto issue = [&](int s) {
    double* dst = Ts + (size_t)(s & 1) * kSkH * kSkPitch;
    const int a0 = s * kSkH;
    for (int e = tid; e < kSkH * (kSkCols / 2); e += kSkW * 32) {
      const int r = e / (kSkCols / 2), col = 2 * (e % (kSkCols / 2));
      const int row = a0 + r;
      const int bytes = row < bi ? (col + 1 < bj ? 16 : (col < bj ? 8 : 0)) : 0;
      cp_async16(dst + (size_t)r * kSkPitch + col, bytes ? Tc + (size_t)row * b + col : Tc, bytes);
    }
    cp_async_commit();
  };
  issue(0);

  // B fragments of P for phase A: rows col0 + 4 kk + tg, columns 8 nt + g of the group
  double pf[8][2];
#pragma unroll
  for (int kk = 0; kk < 8; ++kk)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      const int row = col0 + 4 * kk + tg, q = grp * 16 + 8 * nt + g;
      pf[kk][nt] = row < bj ? (omega ? omega_entry((uint32_t)t, (uint32_t)row, (uint32_t)q)
                                     : P[pbase + (size_t)q * b + row])
                            : 0.0;
    }
  double za[4][2][2];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) za[m][nt][0] = za[m][nt][1] = 0.0;
  // MODE 2: B fragments of P^T for the residual, P rows col0 + 8 j + g, columns 4 kq + tg
  double pt[4][4];
  double rho = 0.0, fro = 0.0;
  if (MODE == 2) {
#pragma unroll
    for (int kq = 0; kq < 4; ++kq)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int row = col0 + 8 * j + g;
        pt[kq][j] = row < bj ? P[pbase + (size_t)(4 * kq + tg) * b + row] : 0.0;
      }
  }

  for (int s = 0; s < nslab; ++s) {
    cp_async_wait_all();
    __syncthreads();  // slab s visible to all; every warp is done with slab s - 1
    if (s + 1 < nslab) issue(s + 1);
    const double* Tsl = Ts + (size_t)(s & 1) * kSkH * kSkPitch;
    double ya[2][2][2];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) ya[m][nt][0] = ya[m][nt][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk)
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const double a = Tsl[(size_t)(8 * m + g) * kSkPitch + col0 + 4 * kk + tg];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) dmma884(ya[m][nt][0], ya[m][nt][1], a, pf[kk][nt]);
      }
    double* yp = Yp + (size_t)warp * kSkH * kSkYp;
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) yp[(8 * m + g) * kSkYp + 8 * nt + 2 * tg + h] = ya[m][nt][h];
    __syncthreads();
    if (tid < kSkH * 16) {
      const int r = tid >> 4, q = tid & 15;
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < kSkW; ++w) sum += Yp[(size_t)w * kSkH * kSkYp + r * kSkYp + q];
      if (mode == 1) {
        const int row = s * kSkH + r;
        if (row < bi) out[pbase + (size_t)(grp * 16 + q) * b + row] = sum;
      }
      if (MODE != 1) Ys[r * kSkYs + q] = sum;
    }
    if (MODE == 1) continue;
    __syncthreads();
    if (MODE == 2) {
      // E_R[:, strip] = T_R[:, strip] - C_R P[strip, :]^T
      double e[2][4][2];
#pragma unroll
      for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) e[m][j][h] = Tsl[(size_t)(8 * m + g) * kSkPitch + col0 + 8 * j + 2 * tg + h];
#pragma unroll
      for (int kq = 0; kq < 4; ++kq)
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          const double a = -Ys[(8 * m + g) * kSkYs + 4 * kq + tg];
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma884(e[m][j][0], e[m][j][1], a, pt[kq][j]);
        }
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const bool rin = s * kSkH + 8 * m + g < bi;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            if (rin && col0 + 8 * j + 2 * tg + h < bj) {
              const double tv = Tsl[(size_t)(8 * m + g) * kSkPitch + col0 + 8 * j + 2 * tg + h];
              rho = fma(e[m][j][h], e[m][j][h], rho);
              fro = fma(tv, tv, fro);
            }
          }
      }
      continue;
    }
    if constexpr (MODE == 0) {  // the sketch's second product; the other modes left above
#pragma unroll
      for (int kq = 0; kq < kSkH / 4; ++kq) {
        double bf[2];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) bf[nt] = Ys[(4 * kq + tg) * kSkYs + 8 * nt + g];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const double a = Tsl[(size_t)(4 * kq + tg) * kSkPitch + col0 + 8 * m + g];
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) dmma884(za[m][nt][0], za[m][nt][1], a, bf[nt]);
        }
      }
    }
  }
  if (MODE == 2) {
    rho = warp_sum(rho);
    fro = warp_sum(fro);
    __syncthreads();
    if (lane == 0) {
      Yp[warp] = rho;
      Yp[kSkW + warp] = fro;
    }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, f = 0.0;
      for (int w = 0; w < kSkW; ++w) {
        a += Yp[w];
        f += Yp[kSkW + w];
      }
      parts[c] = a;
      fparts[c] = f;
    }
  }
  if (MODE == 0) {
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int col = col0 + 8 * m + g;
      if (col < bj)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
          for (int h = 0; h < 2; ++h) out[pbase + (size_t)(grp * 16 + 8 * nt + 2 * tg + h) * b + col] = za[m][nt][h];
    }
  }
}

// ----------------------------------------------------------------------------------------
// P <- Q of the Householder QR of Z (bj x k); the panel is staged in shared memory.
__global__ void __launch_bounds__(1024) k_orth(double* TLR_RESTRICT Z, int n, int b, int k, int ldp,
                                             int tile_base, const int* TLR_RESTRICT tj,
                                             const int* TLR_RESTRICT need, double* TLR_RESTRICT gscratch,
                                             int in_smem, const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const int c = blockIdx.x;
  if (!need[c]) return;
  const int bj = min(b, n - tj[tile_at(status, tile_base + c)] * b);
  const int ke = min(k, bj);  // a tile narrower than k gets a full basis and zero columns
  if (threadIdx.x == 0) add_work(status, 3, 4.0 * bj * ke * ke, 16.0 * bj * k);
  extern __shared__ double smem[];
  double* red = smem;         // 33
  double* tau = smem + 40;    // k
  double* A = tau + 136;      // bj x k (ld bj) when it fits, else global scratch
  const size_t pbase = (size_t)c * b * ldp;
  double* W = in_smem ? A : gscratch + pbase;
  for (int e = threadIdx.x; e < bj * ke; e += blockDim.x) {
    const int row = e % bj, q = e / bj;
    W[(size_t)q * bj + row] = Z[pbase + (size_t)q * b + row];
  }
  __syncthreads();
  cta_geqr2(W, bj, bj, ke, tau, red);
  cta_org2r(W, bj, bj, ke, tau);
  for (int e = threadIdx.x; e < bj * k; e += blockDim.x) {
    const int row = e % bj, q = e / bj;
    Z[pbase + (size_t)q * b + row] = (q < ke) ? W[(size_t)q * bj + row] : 0.0;
  }
}

// ----------------------------------------------------------------------------------------
// The same orthonormalisation for k = 16 and 32 (8 or 16 warps) and tiles up to 512 rows with the
// panel in registers: warp w holds columns 2w and 2w + 1, lane l rows l + 32 i (i < 16).  Per column c the owning
// warp forms the reflector (LAPACK dlarfg convention, as cta_geqr2) and publishes it to shared
// memory; every warp applies it to its own later columns (one warp reduction per column), so a
// column costs two block barriers and no shared-memory traffic for the panel itself.  Q is formed
// backwards from the reflectors kept in the owners' registers (dorg2r order, as cta_org2r).
constexpr int kOrCpw = 2;   // columns per warp
constexpr int kOrRpl = 16;  // rows per lane (tiles up to 512 rows)

// One column of k_orth_reg's QR: the reflector of column cc, held by this warp as its column
// `sel` (lane l rows l + 32 i), in the dlarfg convention; v (unit at cc) to vs, tau to taus[cc],
// beta on the diagonal.  The column is picked by value (sel ? a[1] : a[0]) so that the register
// panel is never indexed at run time.
__device__ __forceinline__ void orth_reflector(double (&a)[kOrCpw][kOrRpl], int sel, int cc, int bj, double* vs,
                                               double* taus) {
  const int lane = threadIdx.x & 31;
  double s2 = 0.0, xa = 0.0;
#pragma unroll
  for (int i = 0; i < kOrRpl; ++i) {
    const int row = lane + 32 * i;
    const double x = sel ? a[1][i] : a[0][i];
    if (row > cc && row < bj) s2 = fma(x, x, s2);
    if (i == cc / 32) xa = x;
  }
  const double sig2 = warp_sum(s2);
  const double alpha = __shfl_sync(0xffffffffu, xa, cc % 32);
  double beta, tc, scale;
  if (sig2 == 0.0) { tc = 0.0; beta = alpha; scale = 1.0; }
  else {
    beta = -copysign(sqrt(alpha * alpha + sig2), alpha);
    tc = (beta - alpha) / beta;
    scale = 1.0 / (alpha - beta);
  }
#pragma unroll
  for (int i = 0; i < kOrRpl; ++i) {
    const int row = lane + 32 * i;
    const double x = sel ? a[1][i] : a[0][i];
    double v = 0.0, y = x;
    if (row > cc && row < bj) {
      y = tc != 0.0 ? x * scale : x;
      v = y;
    } else if (row == cc) {
      v = 1.0;
      y = beta;
    }
    if (sel) a[1][i] = y; else a[0][i] = y;
    vs[row] = v;
  }
  if (lane == 0) taus[cc] = tc;
}

// The reflector of column cc (kept below its diagonal in column `sel`) back to vs for Q.
__device__ __forceinline__ void orth_publish(const double (&a)[kOrCpw][kOrRpl], int sel, int cc, int bj, double* vs) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < kOrRpl; ++i) {
    const int row = lane + 32 * i;
    const double x = sel ? a[1][i] : a[0][i];
    vs[row] = (row > cc && row < bj) ? x : (row == cc ? 1.0 : 0.0);
  }
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 16 / WARPS) k_orth_reg(double* TLR_RESTRICT Z, int n, int b, int ldp,
                                                                   int tile_base, const int* TLR_RESTRICT tj,
                                                                   const int* TLR_RESTRICT need,
                                                                   const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const int c = blockIdx.x;
  if (!need[c]) return;
  constexpr int k = WARPS * kOrCpw;
  const int bj = min(b, n - tj[tile_at(status, tile_base + c)] * b);
  const int ke = min(k, bj);  // a tile narrower than k gets a full basis and zero columns
  if (threadIdx.x == 0) add_work(status, 3, 4.0 * bj * ke * ke, 16.0 * bj * k);
  __shared__ double vs[32 * kOrRpl];  // the current reflector, zero above its pivot
  __shared__ double taus[k];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t pbase = (size_t)c * b * ldp;
  double a[kOrCpw][kOrRpl];
#pragma unroll
  for (int j = 0; j < kOrCpw; ++j) {
    const int col = warp * kOrCpw + j;
#pragma unroll
    for (int i = 0; i < kOrRpl; ++i) {
      const int row = lane + 32 * i;
      a[j][i] = (col < ke && row < bj) ? Z[pbase + (size_t)col * b + row] : 0.0;
    }
  }
  // ---- QR: reflectors below the diagonal of their columns, R on and above it
  for (int cc = 0; cc < ke; ++cc) {
    if (warp == cc / kOrCpw) {
      orth_reflector(a, cc % kOrCpw, cc, bj, vs, taus);
    }
    __syncthreads();
    const double tc = taus[cc];
#pragma unroll
    for (int j = 0; j < kOrCpw; ++j) {
      const int col = warp * kOrCpw + j;
      if (col > cc && col < ke) {
        double w = 0.0;
#pragma unroll
        for (int i = 0; i < kOrRpl; ++i) w = fma(vs[lane + 32 * i], a[j][i], w);
        w = warp_sum(w) * tc;
#pragma unroll
        for (int i = 0; i < kOrRpl; ++i) a[j][i] = fma(-w, vs[lane + 32 * i], a[j][i]);
      }
    }
    __syncthreads();  // vs is rewritten for the next column
  }
  // ---- Q = H_0 ... H_{ke-1} [I; 0], backwards
  for (int cc = ke - 1; cc >= 0; --cc) {
    const double tc = taus[cc];
    if (warp == cc / kOrCpw) {
      orth_publish(a, cc % kOrCpw, cc, bj, vs);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kOrCpw; ++j) {
      const int col = warp * kOrCpw + j;
      if (col > cc && col < ke && tc != 0.0) {
        double w = 0.0;
#pragma unroll
        for (int i = 0; i < kOrRpl; ++i) w = fma(vs[lane + 32 * i], a[j][i], w);
        w = warp_sum(w) * tc;
#pragma unroll
        for (int i = 0; i < kOrRpl; ++i) a[j][i] = fma(-w, vs[lane + 32 * i], a[j][i]);
      }
      if (col == cc) {
#pragma unroll
        for (int i = 0; i < kOrRpl; ++i) {
          const int row = lane + 32 * i;
          a[j][i] = row < cc || row >= bj ? 0.0 : (row == cc ? 1.0 - tc : -tc * vs[row]);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < kOrCpw; ++j) {
    const int col = warp * kOrCpw + j;
#pragma unroll
    for (int i = 0; i < kOrRpl; ++i) {
      const int row = lane + 32 * i;
      if (row < bj) Z[pbase + (size_t)col * b + row] = col < ke ? a[j][i] : 0.0;
    }
  }
}

// ----------------------------------------------------------------------------------------
// Residual of the projection, per column block of 64: parts[c][blk] = sum (T - C P^T)^2 over
// the block, fparts[c][blk] = sum T^2 over the block.  Element-wise, no cancellation.
__global__ void __launch_bounds__(256) k_resid(const double* TLR_RESTRICT T, int n, int b, int k, int ldp,
                                              int tile_base, const int* TLR_RESTRICT ti,
                                              const int* TLR_RESTRICT tj, const int* TLR_RESTRICT need,
                                              const double* TLR_RESTRICT P, const double* TLR_RESTRICT C,
                                              double* TLR_RESTRICT parts, double* TLR_RESTRICT fparts,
                                              int nblk, const int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const int c = blockIdx.x, blk = blockIdx.y;
  if (!need[c]) return;
  const int t = tile_at(status, tile_base + c);
  const int bi = min(b, n - ti[t] * b), bj = min(b, n - tj[t] * b);
  const int q0 = blk * 64;
  if (q0 >= bj) {
    if (threadIdx.x == 0) { parts[c * nblk + blk] = 0.0; fparts[c * nblk + blk] = 0.0; }
    return;
  }
  const int qn = min(64, bj - q0);
  if (threadIdx.x == 0) add_work(status, 5, 2.0 * bi * qn * (k + 1), 8.0 * ((double)bi * qn + (bi + qn) * k));
  extern __shared__ double smem[];
  double* Pb = smem;              // [64][k+1]  P rows q0..q0+63
  double* Cs = Pb + 64 * (k + 1); // [16][k+1]  C rows of the strip
  double* red = Cs + 16 * (k + 1);
  const size_t pbase = (size_t)c * b * ldp;
  for (int e = threadIdx.x; e < 64 * k; e += 256) {
    const int r = e % 64, q = e / 64;
    Pb[r * (k + 1) + q] = (r < qn) ? P[pbase + (size_t)q * b + q0 + r] : 0.0;
  }
  const double* Tc = T + (size_t)c * b * b;
  double acc = 0.0, facc = 0.0;
  const int col = threadIdx.x & 63, rsub = threadIdx.x >> 6;  // 4 row lanes x 64 columns
  for (int a0 = 0; a0 < bi; a0 += 16) {
    const int hrows = min(16, bi - a0);
    __syncthreads();
    for (int e = threadIdx.x; e < 16 * k; e += 256) {
      const int r = e % 16, q = e / 16;
      Cs[r * (k + 1) + q] = (r < hrows) ? C[pbase + (size_t)q * b + a0 + r] : 0.0;
    }
    __syncthreads();
    if (col < qn) {
      // rows rsub, rsub + 4, rsub + 8, rsub + 12 of the strip as four independent chains (each
      // element is still T - sum_q C P in q order; rows past the strip contribute nothing)
      double tv[4], sv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = rsub + 4 * u;
        tv[u] = r < hrows ? Tc[(size_t)(a0 + r) * b + q0 + col] : 0.0;
        sv[u] = tv[u];
      }
      const double* pr = Pb + col * (k + 1);
#pragma unroll 4
      for (int q = 0; q < k; ++q) {
        const double pq = pr[q];
#pragma unroll
        for (int u = 0; u < 4; ++u) sv[u] = fma(-Cs[(rsub + 4 * u) * (k + 1) + q], pq, sv[u]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (rsub + 4 * u < hrows) {
          acc = fma(sv[u], sv[u], acc);
          facc = fma(tv[u], tv[u], facc);
        }
      }
    }
  }
  const double tot = block_sum(acc, red);
  const double ftot = block_sum(facc, red);
  if (threadIdx.x == 0) { parts[c * nblk + blk] = tot; fparts[c * nblk + blk] = ftot; }
}

// ----------------------------------------------------------------------------------------
// Rank decision and output of the truncated pair for every tile still in need.
__global__ void __launch_bounds__(1024) k_finalize(int n, int b, int k, int ldp, int cap, int margin,
                                                 int tile_base, const int* TLR_RESTRICT ti,
                                                 const int* TLR_RESTRICT tj, int* TLR_RESTRICT need,
                                                 const double* TLR_RESTRICT P, const double* TLR_RESTRICT C,
                                                 const double* TLR_RESTRICT parts,
                                                 const double* TLR_RESTRICT fparts, int nblk,
                                                 double* TLR_RESTRICT gscratch, double* TLR_RESTRICT gsv,
                                                 double* TLR_RESTRICT Uo,
                                                 double* TLR_RESTRICT Vo, int* TLR_RESTRICT rank,
                                                 int last_level, int w_in_smem, int* TLR_RESTRICT rlog,
                                                 double* TLR_RESTRICT tail0, double* TLR_RESTRICT fro0,
                                                 int* TLR_RESTRICT blog, int* TLR_RESTRICT status) {
  if (*status != 0) return;
  const EvalParams& prm = *eval_params(status);
  const int rule_fixed = prm.rule_fixed, rmode = prm.rmode, round_store = prm.round_store;
  const double thr_rel = prm.thr_rel, thr_abs = prm.thr_abs;
  const int c = blockIdx.x;
  if (!need[c]) return;
  const int t = tile_at(status, tile_base + c);
  const int bi = min(b, n - ti[t] * b), bj = min(b, n - tj[t] * b);
  if (threadIdx.x == 0) add_work(status, 6, 4.0 * bi * k * k + 6.0 * 8.0 * k * k * k, 8.0 * (bi + bj) * k);
  extern __shared__ double smem[];
  double* red = smem;             // 33 (+pad)
  double* tau = smem + 40;        // k
  double* sig = tau + 136;        // k
  int* perm = reinterpret_cast<int*>(sig + 136);  // k
  int* iflag = perm + 136;
  int* rsel = iflag + 2;
  double* M = (k <= 64) ? smem + 40 + 136 * 3 + 8 : gsv + (size_t)c * 2 * k * k;  // k x k
  double* Vw = M + k * k;                                                             // k x k
  const size_t pbase = (size_t)c * b * ldp;
  // bi x k copy of C for the QR: in shared memory (ld bi) when it fits, else global scratch (ld b)
  double* W = w_in_smem ? smem + 40 + 136 * 3 + 8 + 2 * (size_t)k * k : gscratch + pbase;
  const int ldw = w_in_smem ? bi : b;
  for (int e = threadIdx.x; e < bi * k; e += blockDim.x) {
    const int row = e % bi, q = e / bi;
    W[(size_t)q * ldw + row] = C[pbase + (size_t)q * b + row];
  }
  __syncthreads();
  const int kk = min(k, bi);
  cta_geqr2(W, ldw, bi, k, tau, red);
  cta_copy_r(W, ldw, bi, k, M, k);
  cta_jacobi_svd(M, k, k, k, Vw, k, sig, perm, iflag);
  if (threadIdx.x == 0) {
    double rho2 = 0.0, fro2 = 0.0;
    for (int q = 0; q < nblk; ++q) { rho2 += parts[c * nblk + q]; fro2 += fparts[c * nblk + q]; }
    double sorted[128];
    for (int q = 0; q < k; ++q) sorted[q] = sig[perm[q]];
    const double thr = rule_fixed ? thr_rel * sqrt(fro2) : thr_abs;
    int r = select_rank(sorted, k, rho2, thr, nullptr);
    if (rmode == kRankReplay) r = rlog[t];  // frozen: the rank recorded at another theta
    const bool exact = (k >= bj) || (k >= bi);
    int out;
    if (r >= 0 && (r <= k - margin || exact)) out = r;
    else if (last_level) out = -2;  // compression limit reached
    else out = -1;                  // redo with a larger k
    if (out >= 0 && out > cap) out = -3;
    if (out >= 0) {  // truncation error ||T - T_r||_F and ||T||_F of the accepted tile
      double acc = rho2;
      for (int q = out; q < k; ++q) acc += sorted[q] * sorted[q];
      tail0[t] = sqrt(acc);
      fro0[t] = sqrt(fro2);
    }
    *rsel = out;
  }
  __syncthreads();
  const int r = *rsel;
  (void)kk;
  if (r == -1) return;
  if (r < 0) {
    if (threadIdx.x == 0) atomicCAS(status, 0, r == -2 ? -5 : -2);
    return;
  }
  // U = C W_r, V = P W_r (columns in descending singular-value order)
  double* Ut = Uo + (size_t)t * b * cap;
  double* Vt = Vo + (size_t)t * b * cap;
  for (int e = threadIdx.x; e < bi * r; e += blockDim.x) {
    const int row = e % bi, q = e / bi;
    const double* w = Vw + (size_t)perm[q] * k;
    double s = 0.0;
    for (int u = 0; u < k; ++u) s = fma(C[pbase + (size_t)u * b + row], w[u], s);
    Ut[(size_t)q * b + row] = s;
  }
  for (int e = threadIdx.x; e < bj * r; e += blockDim.x) {
    const int row = e % bj, q = e / bj;
    const double* w = Vw + (size_t)perm[q] * k;
    double s = 0.0;
    for (int u = 0; u < k; ++u) s = fma(P[pbase + (size_t)u * b + row], w[u], s);
    Vt[(size_t)q * b + row] = s;
  }
  if (round_store) {  // storage rule 'mixed': rounded under the budget left after truncation (17:163-164)
    __syncthreads();
    const int bits = cta_round_pair(Ut, Vt, bi, bj, r, b, thr_abs - tail0[t], red,
                                    rmode == kRankReplay ? blog[t] : 0);
    if (threadIdx.x == 0 && rmode == kRankRecord) blog[t] = bits;
  }
  if (threadIdx.x == 0) {
    rank[t] = r;
    need[c] = 0;
    if (rmode == kRankRecord) rlog[t] = r;
  }
}

// ----------------------------------------------------------------------------------------
// launchers
int launch_gen_offdiag(const double* xy, int n, int b, int tile_base, const int* ti, const int* tj,
                       double* T, int nchunk, const int* status, cudaStream_t s) {
  dim3 grid((unsigned)((b * b + 1023) / 1024), (unsigned)nchunk);
  k_gen_offdiag<<<grid, 256, 0, s>>>(xy, n, b, tile_base, ti, tj, T, status);
  return (int)cudaGetLastError();
}

static size_t sketch_smem(int b, int H) { return ((size_t)b * 16 + (size_t)H * (b + 1) + 256 * 4 + H * 16) * 8; }

int launch_sketch(const double* T, int n, int b, int k, int tile_base, const int* ti, const int* tj,
                  const int* need, const double* P, double* out, int ldp, int omega, int mode, int nchunk,
                  const int* status, cudaStream_t s) {
  dim3 grid((unsigned)nchunk, (unsigned)(k / 16));
  if (b <= kSkCols && b % 2 == 0) {  // 16-byte aligned rows: the tensor-core form
    const size_t sm = sketch_mma_smem();
    if (mode == 0) {
      cudaFuncSetAttribute(k_sketch_mma<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_sketch_mma<0><<<grid, kSkW * 32, sm, s>>>(T, n, b, tile_base, ti, tj, need, P, out, ldp, omega, nullptr,
                                                  nullptr, status);
    } else {
      cudaFuncSetAttribute(k_sketch_mma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_sketch_mma<1><<<grid, kSkW * 32, sm, s>>>(T, n, b, tile_base, ti, tj, need, P, out, ldp, omega, nullptr,
                                                  nullptr, status);
    }
  } else if (b <= 512) {
    const size_t sm = sketch_smem(b, 16);
    cudaFuncSetAttribute(k_sketch<16, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_sketch<16, 2><<<grid, 256, sm, s>>>(T, n, b, k, tile_base, ti, tj, need, P, out, ldp, omega, mode, status);
  } else {
    const size_t sm = sketch_smem(b, 8);
    cudaFuncSetAttribute(k_sketch<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_sketch<8, 4><<<grid, 256, sm, s>>>(T, n, b, k, tile_base, ti, tj, need, P, out, ldp, omega, mode, status);
  }
  return (int)cudaGetLastError();
}

bool project_resid_fused(int b, int k) { return k == 16 && b <= kSkCols && b % 2 == 0; }

int launch_project_resid(const double* T, int n, int b, int tile_base, const int* ti, const int* tj,
                         const int* need, const double* P, double* C, int ldp, double* parts, double* fparts,
                         int nchunk, const int* status, cudaStream_t s) {
  if (!project_resid_fused(b, 16)) return (int)cudaErrorInvalidValue;
  const size_t sm = sketch_mma_smem();
  cudaFuncSetAttribute(k_sketch_mma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_sketch_mma<2><<<dim3((unsigned)nchunk, 1), kSkW * 32, sm, s>>>(T, n, b, tile_base, ti, tj, need, P, C, ldp, 0,
                                                                   parts, fparts, status);
  return (int)cudaGetLastError();
}

int launch_orth(double* Z, int n, int b, int k, int ldp, int tile_base, const int* tj, const int* need,
                double* gscratch, int nchunk, const int* status, cudaStream_t s) {
  if (k == 16 && b <= 32 * kOrRpl) {  // panel in registers
    k_orth_reg<8><<<nchunk, 256, 0, s>>>(Z, n, b, ldp, tile_base, tj, need, status);
    return (int)cudaGetLastError();
  }
  if (k == 32 && b <= 32 * kOrRpl) {
    k_orth_reg<16><<<nchunk, 512, 0, s>>>(Z, n, b, ldp, tile_base, tj, need, status);
    return (int)cudaGetLastError();
  }
  size_t sm = (40 + 136) * 8;
  const int in_smem = (size_t)b * k * 8 <= 160 * 1024;
  if (in_smem) sm += (size_t)b * k * 8;
  cudaFuncSetAttribute(k_orth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  // the wide levels hold few tiles, each a long chain of column steps: four times the warps per
  // step there
  k_orth<<<nchunk, k >= 32 ? 1024 : 256, sm, s>>>(Z, n, b, k, ldp, tile_base, tj, need, gscratch, in_smem, status);
  return (int)cudaGetLastError();
}

int launch_resid(const double* T, int n, int b, int k, int ldp, int tile_base, const int* ti, const int* tj,
                 const int* need, const double* P, const double* C, double* parts, double* fparts, int nblk,
                 int nchunk, const int* status, cudaStream_t s) {
  const size_t sm = ((size_t)64 * (k + 1) + 16 * (k + 1) + 40) * 8;
  cudaFuncSetAttribute(k_resid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 grid((unsigned)nchunk, (unsigned)nblk);
  k_resid<<<grid, 256, sm, s>>>(T, n, b, k, ldp, tile_base, ti, tj, need, P, C, parts, fparts, nblk, status);
  return (int)cudaGetLastError();
}

int launch_finalize(int n, int b, int k, int ldp, int cap, int margin, int tile_base, const int* ti, const int* tj,
                    int* need, const double* P, const double* C, const double* parts, const double* fparts,
                    int nblk, double* gscratch, double* gsv, double* U, double* V, int* rank, int last_level,
                    int nchunk, int* rlog, double* tail0, double* fro0, int* blog, int* status, cudaStream_t s) {
  size_t sm = (40 + 136 * 3 + 8 + (k <= 64 ? 2 * (size_t)k * k : 0)) * 8;
  const int w_in_smem = k <= 64 && (size_t)b * k * 8 <= 160 * 1024;
  if (w_in_smem) sm += (size_t)b * k * 8;
  cudaFuncSetAttribute(k_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_finalize<<<nchunk, k >= 32 ? 1024 : 256, sm, s>>>(n, b, k, ldp, cap, margin, tile_base, ti, tj, need, P, C, parts,
                                                      fparts, nblk, gscratch, gsv, U, V, rank, last_level,
                                                      w_in_smem, rlog, tail0, fro0, blog, status);
  return (int)cudaGetLastError();
}

}  // namespace tlr
