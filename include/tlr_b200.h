/*
 * C ABI of the B200 adaptive tile-low-rank (TLR) Gaussian-process log-likelihood.
 *
 * The reference (marysalvana/adaptive-tlr-pilots) has no FFI: its scripts load
 * codes/11_tlr_rank_rules.py and codes/17_tlr_cholesky_pilot.py by file path and call Python
 * functions.  Each entry point below replaces one of those calls; the comment on each names
 * the reference interface (path:line) it stands in for.  The Python package
 * adaptive_tlr_pilots_b200 binds these symbols with ctypes and presents the reference's call
 * surface on top of them.
 *
 * Conventions
 *   - plain C types only; device pointers are CUDA device addresses, host pointers are host
 *     addresses; sizes are element counts;
 *   - every function returns a status: 0 on success, > 0 only where documented (a factorization
 *     that is not positive definite), < 0 on error, with a message in tlr_last_error();
 *   - nothing aborts, nothing throws; no call prints;
 *   - a plan owns all of its device memory (allocated once, at creation); a plan is used by one
 *     host thread at a time; work is issued on the plan's stream.
 */
#ifndef TLR_B200_H
#define TLR_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* rank rules: codes/17_tlr_cholesky_pilot.py:149-150 */
#define TLR_RULE_FIXED 0    /* relative Frobenius tolerance eps per tile */
#define TLR_RULE_ADAPTIVE 1 /* absolute budget tau * b * sigma2 * eta / N */
#define TLR_RULE_MIXED 2    /* adaptive ranks, every stored factor pair rounded to the fewest bits
                               (FP8 / FP16 / FP32 / FP64) that fit the budget left after
                               truncation: codes/17_tlr_cholesky_pilot.py:33-82, 145-148 */

/* status codes */
#define TLR_OK 0
#define TLR_ERR_ARG (-1)          /* invalid argument */
#define TLR_ERR_RANK_CAP (-2)     /* a tile rank exceeded the plan's rank capacity */
#define TLR_ERR_CUDA (-3)         /* CUDA runtime error */
#define TLR_ERR_NOMEM (-4)        /* device allocation failed */
#define TLR_ERR_COMPRESS (-5)     /* a tile needed more than the largest sketch width */
#define TLR_ERR_NOT_READY (-6)    /* tlr_set_data has not been called */
#define TLR_ERR_TIMEOUT (-7)      /* a bounded device wait gave up (the kernel freed its resources) */

typedef struct tlr_plan tlr_plan;

/* Per-evaluation statistics, the `info` dict of codes/17_tlr_cholesky_pilot.py:167, 175, 206-209. */
typedef struct {
  int completed;            /* 1 when every diagonal tile factorized */
  int failed_at;            /* first diagonal tile that is not positive definite, or -1 */
  long long stored_sigma;   /* stored values of the compressed covariance (17:154-167) */
  int max_rank_sigma;
  long long stored_factor;  /* stored values of the factor (17:206) */
  double mean_rank_factor;
  int max_rank_factor;
  double logdet;            /* 2 sum log diag L_kk */
  double quad;              /* z^T z, z = L^{-1} y */
} tlr_info;

/* Outputs of the assembled-matrix rule, codes/11_tlr_rank_rules.py:74-108 truncate_tiles. */
typedef struct {
  long long stored;   /* dense diagonal tiles + 2 b_max r_ij per off-diagonal tile (11:83, 101) */
  double max_rel;     /* max over tiles of ||T - T_r||_F / ||T||_F */
  double max_abs;     /* max over tiles of ||T - T_r||_F */
  double fro_err;     /* ||Sigma - Sigma^TLR||_F = sqrt(2 sum ||T - T_r||_F^2) */
  int max_rank;
} tlr_tile_stats;

/* Create a plan for N sites in tiles of b (the last tile may be short, as
 * codes/11_tlr_rank_rules.py:69-71 tile_bounds), with room for `cap` columns per off-diagonal
 * factor.  stream may be NULL (the legacy default stream).  Allocates all device memory. */
int tlr_plan_create(tlr_plan** plan, int n, int b, int cap, int device, void* stream);
void tlr_plan_destroy(tlr_plan* plan);

/* Morton (Z-order) permutation of n points (device xy, n x 2, row-major) into device perm
 * (n int64): replaces morton_order, codes/11_tlr_rank_rules.py:40-53 (order = bits per axis). */
int tlr_morton_order(const double* xy_dev, int n, int order, long long* perm_dev, void* stream);

/* Allocation-free form of tlr_morton_order for callers that may not allocate device memory
 * during the call (a framework's caching allocator owns the device memory, a service loop that
 * must not allocate after start-up, ...).  No counterpart in the reference.  Same inputs,
 * outputs and result as tlr_morton_order; the working memory is an 8.5 MiB array inside the
 * library's device image (held by every GPU that loads the library until the process exits),
 * so n <= 1,048,576 and order <= 10, otherwise TLR_ERR_ARG.  Every call looks up the array's
 * device address (cheap, no allocation).  With CUDA's lazy module loading (the default), the
 * array itself comes into existence at the first call on each device, which does take device
 * memory once: make that first call at start-up, before any stream capture and before another
 * framework's caching allocator has taken the device's memory.  The work is queued
 * on `stream` and the call returns without waiting.  All calls share the one array: calls
 * whose work can overlap on the GPU (different streams, or different host threads) race, so
 * serialise them, for example on one stream. */
int tlr_morton_order_noalloc(const double* xy_dev, int n, int order, long long* perm_dev, void* stream);

/* Load Morton-ordered sites (device, n x 2 row-major) and observations (device, n) into the
 * plan (copied; the caller keeps ownership).  The reference passes S and y to every call of
 * tlr_loglik (codes/17_tlr_cholesky_pilot.py:259); here they are loaded once. */
int tlr_set_data(tlr_plan* plan, const double* xy_dev, const double* y_dev);

/* Log-likelihood at theta = (sigma2, range, eta) with rule TLR_RULE_FIXED (value = eps) or
 * TLR_RULE_ADAPTIVE (value = tau): replaces tlr_loglik, codes/17_tlr_cholesky_pilot.py:259-266
 * (tlr_cholesky 137-215 and tlr_forward 230-240 inside).
 * Returns 0 on success, k + 1 when diagonal tile k is not positive definite (the reference's
 * (None, None, {completed: False, failed_at: k}), 17:172-176), < 0 on error.
 * loglik, info, factor_ranks and sigma_ranks are host pointers and may be NULL.
 * factor_ranks receives nB (nB - 1) / 2 ranks in the reference's L_off order (for k, for i > k,
 * 17:207); sigma_ranks the initial ranks in the order (for i, for j < i) (17:155-166). */
int tlr_loglik(tlr_plan* plan, const double theta[3], int rule, double value, double* loglik, tlr_info* info,
               int* factor_ranks, int* sigma_ranks);

/* Log-likelihood and its gradient in theta = (sigma2, range, eta), ranks frozen at theta.
 * No counterpart in the reference (it has no gradient code; its only derivatives are central
 * finite differences, codes/15_pilot_standard_errors.py:21-31).  grad = 1/2 alpha^T dSigma alpha
 * - 1/2 tr(Sigma_t^{-1} dSigma) with Sigma_t = L L^T the TLR factor, alpha = Sigma_t^{-1} y, the
 * inverse tiles from a selected inversion on the factor (the blocked Cholesky adjoint with the
 * truncations passed through) and dSigma regenerated from the sites.  Same return convention as
 * tlr_loglik; grad (host, 3 doubles) is written only on success. */
int tlr_loglik_grad(tlr_plan* plan, const double theta[3], int rule, double value, double* loglik, double* grad,
                    tlr_info* info, int* factor_ranks, int* sigma_ranks);

/* Batched log-likelihood and gradient: plans[q] evaluates thetas[3q .. 3q+2] (count plans, all
 * distinct, same device, each with its own stream and its data loaded).  Every forward pass is
 * queued before any is waited on, then every backward pass likewise, so the GPU overlaps the
 * plans' latency-bound factorization steps (a batch of MCMC chains or optimizer restarts shares
 * one call).  loglik[q] (NaN when not PD), grad[3q .. 3q+2] (when status[q] == 0) and status[q]
 * (0 ok, k + 1 when diagonal tile k is not positive definite) are host arrays; loglik, grad and
 * status may be NULL.  Returns 0 when every evaluation ran, < 0 on an error of any of them.  No
 * counterpart in the reference (its MCMC evaluates one chain at a time,
 * codes/19_tlr_mcmc_gpu.py:170-202). */
int tlr_loglik_grad_batch(tlr_plan* const* plans, int count, const double* thetas, int rule, double value,
                          double* loglik, double* grad, int* status);

/* The assembled-matrix rule: every off-diagonal tile of Sigma(theta) truncated under the rule
 * (the plan's initial compression, the reference's ranks), with the reference's statistics in
 * `stats` and the per-tile ranks in `ranks` (ntiles, order (i, j < i); may be NULL).  When K_dev
 * is not NULL, Sigma^TLR is written there densely (N x N FP64 on the plan's device, leading
 * dimension ldk >= N; symmetric, so either storage order): the diagonal tiles exact, every
 * off-diagonal tile U V^T and its transpose.  Replaces truncate_tiles / make_cov,
 * codes/11_tlr_rank_rules.py:74-108, 121-126 (whose input is the dense K; here the tiles are
 * generated from the sites), and the truncation of codes/19_tlr_mcmc_gpu.py:51-123.  Leaves no
 * factor in the plan.  Tiles per side (N / b) at most 361. */
int tlr_truncate_tiles(tlr_plan* plan, const double theta[3], int rule, double value, double* K_dev,
                       long long ldk, tlr_tile_stats* stats, int* ranks);

/* The same evaluation with HOST sites and observations (Morton-ordered), copied to the device
 * inside the call: the end-to-end form of tlr_loglik for callers that hold numpy arrays. */
int tlr_loglik_host(tlr_plan* plan, const double* xy_host, const double* y_host, const double theta[3], int rule,
                    double value, double* loglik, tlr_info* info, int* factor_ranks, int* sigma_ranks);

/* Triangular solves with the factor left by the last successful evaluation of the plan, for m
 * right-hand sides in place (x: device, n x m, column-major, ld n): trans 0 solves L X = B
 * (replaces tlr_forward, codes/17_tlr_cholesky_pilot.py:230-240), trans 1 solves L^T X = Z
 * (tlr_backward, 17:243-256).  Together they give Sigma_t^{-1} B for kriging (tlr_predict,
 * 17:269-276).  TLR_ERR_NOT_READY when the plan holds no completed factorization. */
int tlr_factor_solve(tlr_plan* plan, double* x_dev, int m, int trans);

/* Y = L Z with the factor of the last successful evaluation (z, y: device, n x m, column-major,
 * distinct): replaces tlr_matvec_L, codes/17_tlr_cholesky_pilot.py:218-227, with which the
 * reference simulates fields too large for a dense factor (17:326-339). */
int tlr_factor_matvec(tlr_plan* plan, const double* z_dev, double* y_dev, int m);

/* Copy factor pieces to the host for checking: the dense lower factor of diagonal tile k
 * (bk x bk, column-major) or the (U, V) pair of off-diagonal tile (i, j), i > j (b_i x r and
 * b_j x r, column-major, r = *rank).  Valid after a successful tlr_loglik. */
int tlr_get_diag_tile(tlr_plan* plan, int k, double* out_host);
int tlr_get_offdiag_tile(tlr_plan* plan, int i, int j, double* u_host, double* v_host, int* rank);

/* Arithmetic of a plan.  TLR_PRECISION_FP64 (default): every step in FP64, the parity path.
 * TLR_PRECISION_MIXED: the backward pass's GEMMs on the tensor cores as split TF32 (3xTF32, FP32
 * accumulation); FP64 kept for the forward factorization, thresholds, POTRF and all
 * accumulations of log det, quadratic form and gradient.  No reference counterpart (the
 * reference is FP64 throughout). */
#define TLR_PRECISION_FP64 0
#define TLR_PRECISION_MIXED 1
int tlr_plan_set_precision(tlr_plan* plan, int mode);

/* Rank map of later evaluations on the plan.  TLR_RANKS_RULE: the rule picks every rank (the
 * reference's behaviour).  TLR_RANKS_RECORD: the rule picks, and every rank it picks (each
 * initial compression, codes/17_tlr_cholesky_pilot.py:163, and each recompression, 17:203) is
 * recorded in the plan.  TLR_RANKS_REPLAY: the recorded ranks replace the rule's choices (frozen
 * ranks: the TLR log-likelihood as a smooth function of theta, for central differences and the
 * ranks-frozen gradient).  Replay needs a recorded evaluation of the same rule on the same data.
 * No counterpart in the reference, whose finite-difference Hessian
 * (codes/15_pilot_standard_errors.py:21-31) lets the rule re-pick the ranks at every point. */
/* Storage of the factor left by the last completed evaluation: bits[q] (8, 16, 32 or 64) of
 * every off-diagonal factor tile in the reference's L_off order (for k, for i > k), and the stored
 * bytes (dense FP64 diagonal tiles + 2 b_i r_ik bits / 8 per off-diagonal tile).  Replaces the
 * precision bookkeeping of rule 'mixed', codes/17_tlr_cholesky_pilot.py:38, 184, 210-214 (PREC_OF,
 * stored_factor_bytes, precision_mix_factor_tiles); every tile is 64 bits under the other rules.
 * bits and stored_bytes are host pointers and may be NULL.  TLR_ERR_NOT_READY without a factor. */
int tlr_factor_storage(tlr_plan* plan, int* bits, long long* stored_bytes);

#define TLR_RANKS_RULE 0
#define TLR_RANKS_RECORD 1
#define TLR_RANKS_REPLAY 2
int tlr_plan_rank_map(tlr_plan* plan, int mode);

/* The plan's rank map on the host, to keep frozen ranks across plans or processes: the number of
 * recorded ranks (initial tiles, then every step's trailing pairs) is tlr_plan_rank_map_size(plan);
 * ranks holds that many, bits (rule 'mixed': the storage bits chosen at each of those roundings,
 * then at each panel solve, one per tile) that many plus nB (nB - 1) / 2.  upload = 0 copies the map
 * out, 1 copies it in (a later TLR_RANKS_REPLAY evaluation uses it); either pointer may be NULL.
 * No counterpart in the reference. */
long long tlr_plan_rank_map_size(const tlr_plan* plan);
int tlr_plan_rank_map_io(tlr_plan* plan, int* ranks, int* bits, long long count, int upload);

/* Kernel kinds counted by tlr_plan_kernel_stats (launches issued by the plan's evaluations). */
#define TLR_K_FILL 0
#define TLR_K_GEN 1        /* off-diagonal tile generation */
#define TLR_K_SKETCH 2     /* Z = T^T (T P) */
#define TLR_K_ORTH 3       /* Householder orthonormalisation of the sketch */
#define TLR_K_PROJECT 4    /* C = T P */
#define TLR_K_RESID 5      /* ||T - C P^T||_F^2 */
#define TLR_K_FINALIZE 6   /* rank decision + truncated pair */
#define TLR_K_DIAG 7       /* diagonal tile generation + deferred updates */
#define TLR_K_POTRF 8      /* diagonal Cholesky + forward-solve block */
#define TLR_K_TRSM 9       /* panel solve */
#define TLR_K_RECOMPRESS 10 /* Schur update + recompression */
#define TLR_K_FINISH 11
#define TLR_K_BWD_GEMM 12   /* backward: batched GEMMs of the selected inversion */
#define TLR_K_TRI_INV 13    /* backward: inverses of the diagonal factor tiles */
#define TLR_K_BWD_COPY 14   /* backward: panel gathers */
#define TLR_K_ALPHA 15      /* backward: TLR solve alpha = Sigma^{-1} y */
#define TLR_K_DTRACE 16     /* backward: dSigma generation + contraction */
#define TLR_K_GRAD_FINISH 17
#define TLR_NKINDS 18

/* Covariance smoothness for the plan's next evaluations: nu = 1.5 (Matern 3/2, the default,
 * codes/11_tlr_rank_rules.py:35-37) or 2.5 (Matern 5/2, (1 + x + x^2/3) e^{-x}, x = sqrt(5) h /
 * range: codes/24_screening_stress.py:30-47, which patches it into the TLR Cholesky of 17).
 * Other values: TLR_ERR_ARG.  Applies to tile generation, the diagonal tiles and dSigma of the
 * gradient. */
int tlr_plan_set_kernel(tlr_plan* plan, double nu);

/* Profiling: when on, every launch is bracketed by CUDA events on the plan's stream and the
 * per-kind device time is accumulated (no effect on results); on < 0 brackets only the launches
 * of kernel kind -on - 1 (the order of tlr_plan_kernel_stats).  No reference counterpart. */
int tlr_plan_set_profiling(tlr_plan* plan, int on);

/* CUDA graphs (default on): the forward pass of an evaluation (compression, factorization and the
 * forward solve, about 1,000 launches at N = 50,000, b = 500) is captured once per precision on a
 * private stream and replayed on the plan's stream for every theta; theta, the rule and the
 * thresholds reach the kernels through the plan's device control block, written by one launch
 * before each replay.  Off: the same launches are issued one by one.  Results are bit-identical
 * either way; while profiling is on the launches are issued one by one.  No reference counterpart
 * (the reference is a Python loop, codes/17_tlr_cholesky_pilot.py:259-266). */
int tlr_plan_set_graphs(tlr_plan* plan, int on);

/* Block-row cyclic factorization over `world` ranks (codes/13_multigpu_tile_cholesky.py:45-79,
 * tile_cholesky_multi, with the TLR tiles and rank rule of codes/17_tlr_cholesky_pilot.py:137-215).
 * A partitioned plan holds block rows i with i % world == rank: it compresses their tiles and
 * factors them; the diagonal tile of step k lives on rank k % world.  One process (or plan) per
 * rank; the host moves three kinds of device buffers between them and every rank takes the same
 * steps in the same order:
 *
 *   tlr_dist_begin(plan, theta, rule, value)            compression of the rank's tiles; step 0's
 *                                                        diagonal tile on its owner
 *   for k in 0 .. nB-1:
 *     owner of k:  tlr_dist_pack_diag(plan, k, dbuf)     then broadcast dbuf from rank k % world
 *     the others:  tlr_dist_unpack_diag(plan, k, dbuf)   (13:63-66)
 *     tlr_dist_solve_step(plan, k)                       panel solve of the rank's tiles (i, k)
 *     tlr_dist_pack_panel(plan, k, pbuf)                 then all-gather pbuf (length
 *     tlr_dist_unpack_panel(plan, k, gathered)           tlr_dist_buffer_doubles(PANEL, k), rank order)
 *     tlr_dist_update_step(plan, k)                      recompression of the rank's trailing pairs,
 *                                                        and the next diagonal tile on its owner
 *   tlr_dist_pack_sums(plan, sbuf)                       then all-reduce (sum) sbuf
 *   tlr_dist_finish(plan, summed, &loglik, &info, ...)   tlr_loglik's outputs on every rank
 *
 * Every tile is computed by the same kernels as on one plan, so the log-likelihood, ranks and
 * stored sizes are bit-identical to tlr_loglik's (the sums add zeros).  A failure on any rank
 * (a non-positive pivot, a rank past the capacity) travels in the buffers' status word and every
 * rank returns the first one in rank order.  Rules fixed and adaptive; no rank map; a partitioned
 * plan refuses tlr_loglik and the factor-based calls (world = 1 lifts the partition).  Buffer
 * sizes in doubles: tlr_dist_buffer_doubles(plan, TLR_DIST_DIAG | TLR_DIST_PANEL | TLR_DIST_SUMS,
 * k) (PANEL with k < 0: the largest step).  Device buffers, on the plan's stream. */
#define TLR_DIST_DIAG 0
#define TLR_DIST_PANEL 1
#define TLR_DIST_SUMS 2
int tlr_plan_set_partition(tlr_plan* plan, int rank, int world);
long long tlr_dist_buffer_doubles(const tlr_plan* plan, int which, int k);
int tlr_dist_begin(tlr_plan* plan, const double theta[3], int rule, double value);
int tlr_dist_pack_diag(tlr_plan* plan, int k, double* buf);
int tlr_dist_unpack_diag(tlr_plan* plan, int k, const double* buf);
int tlr_dist_solve_step(tlr_plan* plan, int k);
int tlr_dist_pack_panel(tlr_plan* plan, int k, double* buf);
int tlr_dist_unpack_panel(tlr_plan* plan, int k, const double* gathered);
int tlr_dist_update_step(tlr_plan* plan, int k);
int tlr_dist_pack_sums(tlr_plan* plan, double* buf);
int tlr_dist_finish(tlr_plan* plan, const double* sums, double* loglik, tlr_info* info, int* factor_ranks,
                    int* sigma_ranks);
/* Per-kind accumulated device milliseconds (profiling on), launch counts and algorithmic work
 * (FP64 flops and HBM bytes the kernels count for themselves) since the last reset.  Any output
 * pointer may be NULL.  No reference counterpart. */
int tlr_plan_kernel_stats(tlr_plan* plan, double* ms, long long* launches, double* flops, double* bytes, int nkinds,
                          int reset);

/* Self-test of the failure path of the tensor-core kernels' bounded waits (no reference
 * counterpart): one CTA allocates tensor memory and waits, at most `iterations` polls, on an
 * mbarrier phase that nothing completes; it then frees the tensor memory and reports.  Returns
 * TLR_ERR_TIMEOUT when the wait ran out (the expected outcome; the context stays usable), 0 if
 * it did not, < 0 on other errors.  *elapsed_ms (optional): device time of the launch; *limit
 * (optional): the poll limit of the production waits.  Allocates one int on `device`. */
int tlr_selftest_bounded_wait(long long iterations, int device, double* elapsed_ms, long long* limit);

/* Self-test of the backward pass's GEMM kernels (no reference counterpart):
 * C = alpha op(A) op(B) + beta C, column-major, op(X) = X^T when trans != 0, on device pointers
 * of `device`, on the FP64 tensor cores (precision TLR_PRECISION_FP64) or as split TF32 on the
 * tcgen05 tensor cores (TLR_PRECISION_MIXED).  Synchronous; 0 on success, < 0 on errors. */
int tlr_selftest_gemm(int precision, int transA, int transB, int M, int N, int K, double alpha, const double* A,
                      int lda, const double* B, int ldb, double beta, double* C, int ldc, int device);

/* Message of the last error on this thread. */
const char* tlr_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* TLR_B200_H */
