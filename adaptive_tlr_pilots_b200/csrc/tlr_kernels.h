// Host-side launchers of the TLR kernels (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <algorithm>

#include "../../include/tlr_b200.h"

namespace tlr {

// The parameters of one evaluation that change with theta, the rule and the plan's modes.  They
// live in the plan's control block (after the status word and the per-kernel work counters), so
// the forward pass reads them on the device: a launch sequence captured once in a CUDA graph then
// serves every theta.  launch_set_params writes them (kernel arguments, so the host copy is free
// at once) and clears the status word and the counters, ahead of the captured sequence.
struct EvalParams {
  double sigma2, inv_range, nugget;  // covariance: sigma2, 1 / range, sigma2 eta
  double thr_rel, thr_abs;           // rank rule thresholds (17:143-150)
  int rule_fixed;                    // 1: relative rule, 0: absolute budget
  int rmode;                         // rank map: kRankOff / kRankRecord / kRankReplay
  int round_store;                   // storage rule 'mixed': round every stored pair
  int nu5;                           // 0: Matern 3/2, 1: Matern 5/2
  const int* tmap;                   // block-row partition: the tiles this rank compresses (else all)
};
constexpr size_t kControlInts = 4 + 4 * TLR_NKINDS;                       // status, pad, work counters
constexpr size_t kControlBytes = kControlInts * sizeof(int) + sizeof(EvalParams);
__host__ __device__ inline const EvalParams* eval_params(const int* control) {
  return reinterpret_cast<const EvalParams*>(control + kControlInts);
}
// Storage index of the q-th tile the compression visits: every tile in order, or the rank's own
// tiles under a block-row partition.
__device__ __forceinline__ int tile_at(const int* control, int q) {
  const int* m = eval_params(control)->tmap;
  return m ? m[q] : q;
}

// Rank map: every rank the rule picks (initial compression of tile t at rlog[t], recompression of
// trailing pair p of step k at rlog[ntiles + off_k + p]) is recorded, or replayed instead of the
// rule's choice (frozen ranks at another theta).  Under the storage rule 'mixed' the storage bits
// of every rounding go to blog at the same positions, the panel solve's after them (blog[total + t]).
constexpr int kRankOff = 0, kRankRecord = 1, kRankReplay = 2;

// Morton order (codes/11_tlr_rank_rules.py:40-53): stable radix sort of the keys.  `work` holds
// morton_work_words(n, order) unsigned words; perm (n int64) doubles as the sort's second buffer.
size_t morton_work_words(int n, int order);
int launch_morton(const double* xy, int n, int order, unsigned* work, long long* perm, cudaStream_t s);
int launch_gather_sites(const double* xy_in, const double* y_in, const long long* perm, int n, double* xy_out,
                        double* y_out, cudaStream_t s);

// initial compression
int launch_gen_offdiag(const double* xy, int n, int b, int tile_base, const int* ti, const int* tj, double* T,
                       int nchunk, const int* status, cudaStream_t s);
int launch_sketch(const double* T, int n, int b, int k, int tile_base, const int* ti, const int* tj, const int* need,
                  const double* P, double* out, int ldp, int omega, int mode, int nchunk, const int* status,
                  cudaStream_t s);
int launch_orth(double* Z, int n, int b, int k, int ldp, int tile_base, const int* tj, const int* need,
                double* gscratch, int nchunk, const int* status, cudaStream_t s);
// k = 16 and b <= 512 even: projection C = T P and its residual in one pass (parts / fparts get
// one block per tile)
bool project_resid_fused(int b, int k);
int launch_project_resid(const double* T, int n, int b, int tile_base, const int* ti, const int* tj,
                         const int* need, const double* P, double* C, int ldp, double* parts, double* fparts,
                         int nchunk, const int* status, cudaStream_t s);
int launch_resid(const double* T, int n, int b, int k, int ldp, int tile_base, const int* ti, const int* tj,
                 const int* need, const double* P, const double* C, double* parts, double* fparts, int nblk,
                 int nchunk, const int* status, cudaStream_t s);
int launch_finalize(int n, int b, int k, int ldp, int cap, int margin, int tile_base, const int* ti, const int* tj,
                    int* need, const double* P, const double* C, const double* parts, const double* fparts,
                    int nblk, double* gscratch, double* gsv, double* U, double* V, int* rank, int last_level,
                    int nchunk, int* rlog, double* tail0, double* fro0, int* blog, int* status, cudaStream_t s);

// factorization
int launch_diag_build(const double* xy, int n, int b, int k, const double* U, const double* Y, const int* rank,
                      int cap, double* D, const int* status, cudaStream_t s);
int launch_potrf(double* D, int n, int b, int k, double* rhs, double* z, double* ldpart, double* qpart,
                 int* status, cudaStream_t s);
// nbatch tiles, tile q at D + q sD, rhs / z + q sV, ldpart / qpart / status + q sS
int launch_potrf_batched(double* D, int n, int b, int k, double* rhs, double* z, double* ldpart, double* qpart,
                         int* status, int nbatch, size_t sD, size_t sV, int sS, cudaStream_t s);
int launch_trsm(const double* D, int n, int b, int k, int nB, double* U, double* V, double* Wd, double* Y,
                const int* rank, int cap, const double* z, double* rhs, int* prec, int* blog_trsm, int prank,
                int pworld, const int* status, cudaStream_t s);
size_t rc_slot_doubles(int b, int cap);
// every trailing pair of step k; next_pair: a counter that is zero at launch (the CTAs claim
// pairs past the grid through it)
int rc_blocks_per_sm();  // k_recompress CTAs resident per SM
int launch_recompress(int n, int b, int k, int nB, double* U, double* V, int* rank, int cap, double* scratch,
                      size_t slot_doubles, int nslots, int* next_pair, int* rlog_step, int* blog_step, int prank,
                      int pworld, int* status, cudaStream_t s);
// assembled-matrix rule: dense Sigma^TLR from the initial compression (N x N, leading dimension ldk)
int launch_assemble(const double* xy, int n, int b, double sigma2, double inv_range, int nu5, double nugget,
                    const double* U, const double* V, const int* rank, int cap, double* K, long long ldk,
                    const int* status, cudaStream_t s);
int launch_finish(int nB, int n, const double* ldpart, const double* qpart, double* out, const int* status,
                  cudaStream_t s);

// backward pass
struct GemmJob {
  const double* A;
  const double* B;
  double* C;
  double* const* ccol;  // optional per-column destinations of C (then C / ldc are unused)
  int lda, ldb, ldc, M, N, K, transA, transB;
  double alpha, beta;
};
struct CopyJob {
  const double* src;
  double* dst;
  int lds, ldd, rows, cols;
};
int launch_dgemm_batched(const GemmJob* jobs, int njobs, int max_m, int max_n, const int* status, int kind,
                         cudaStream_t s);
// Split-TF32 tensor-core GEMM (tlr_tc.cu).  An operand is first converted once into blocks of
// 128 rows x 16 k (hi then lo TF32 in the UMMA layout, zero-padded), block (row tile t, slice s)
// at dst + (t * nks + s) * 4096 floats, nks = ceil(K / 16).  kcont: element (row, k) of the
// operand at src[row * ld + k], else at src[k * ld + row].
struct SplitJob {
  const double* src;
  float* dst;
  int ld, kcont, rows, K;
};
// per GEMM job: the converted op(A) (M rows) and op(B)^T (N rows), both over K
struct TcOperands {
  const float* a;
  const float* b;
};
// max_blocks: the largest operand's block count
int launch_split_tf32(const SplitJob* jobs, int njobs, int max_blocks, int* status, int kind, cudaStream_t s);
int launch_gemm_tc3(const GemmJob* jobs, const TcOperands* ops, int njobs, int max_m, int max_n, int* status, int kind,
                    cudaStream_t s);
size_t tc_panel_floats(int rows, int K);
int tc_panel_blocks(int rows, int K);
// the bounded-wait self-test (tlr_tc.cu) and the iteration limit of the GEMM's waits
int launch_wait_selftest(long long limit, int* status, cudaStream_t s);
long long tc_wait_limit();
int launch_tri_inv(const double* D, double* Li, int n, int b, int nB, const int* status, cudaStream_t s);
int launch_copy_cols(const CopyJob* jobs, int njobs, const int* status, cudaStream_t s);
int launch_alpha_step(int n, int b, int m, int nB, const double* U, const double* V, const int* rank, int cap,
                      const double* Li, const double* z, double* alpha, double* work, const int* status,
                      cudaStream_t s);
int launch_dtrace_step(const double* xy, int n, int b, int m, int nB, double sigma2, double inv_range, int nu5,
                       double eta, const double* Zbuf, const double* alpha, double* part, const int* status,
                       cudaStream_t s);
int launch_grad_finish(const double* part, long nparts, double* grad, const int* status, cudaStream_t s);

// solves and products with the factor (tlr_solve.cu); column-major n x m, ld n
int launch_factor_solve(const double* D, const double* U, const double* V, const int* rank, int cap, int n, int b,
                        int nB, double* X, int m, int trans, cudaStream_t s);
int launch_factor_matvec(const double* D, const double* U, const double* V, const int* rank, int cap, int n, int b,
                         int nB, const double* Z, double* Y, int m, cudaStream_t s);

// error reporting shared by the library's translation units (message for tlr_last_error)
int set_error(int code, const char* msg);

// small utilities
int launch_fill_int(int* p, int v, int count, cudaStream_t s);
// block-row cyclic factorization: exchange buffers (layouts in tlr_dist.cu)
size_t dist_panel_doubles(int b, int cap, int k, int nB, int pworld);
int launch_dist_pack_diag(const double* D, const double* z, const int* status, int n, int b, int k, double* buf,
                          cudaStream_t s);
int launch_dist_unpack_diag(double* D, double* z, int* status, int n, int b, int k, const double* buf,
                            cudaStream_t s);
int launch_dist_pack_panel(const double* U, const double* V, const int* rank, const int* status, int n, int b, int k,
                           int nB, int cap, int prank, int pworld, double* buf, cudaStream_t s);
int launch_dist_unpack_panel(double* U, double* V, int* rank, int* status, int n, int b, int k, int nB, int cap,
                             int prank, int pworld, const double* gathered, size_t len, cudaStream_t s);
int launch_dist_pack_sums(const double* ldpart, const double* qpart, const int* rank0, const int* ti,
                          const int* status, int nB, int ntiles, int prank, int pworld, double* buf, cudaStream_t s);
int launch_dist_unpack_sums(double* ldpart, double* qpart, int* rank0, int* status, int nB, int ntiles, int pworld,
                            const double* sums, cudaStream_t s);
// control block: zero the status word and the work counters, store the evaluation's parameters
int launch_set_params(int* control, EvalParams prm, cudaStream_t s);

}  // namespace tlr
