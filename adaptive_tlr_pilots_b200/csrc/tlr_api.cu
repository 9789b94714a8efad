// Plan management and the extern "C" entry points declared in include/tlr_b200.h.
//
// One evaluation of the log-likelihood is a fixed sequence of kernel launches on the plan's
// stream (no host synchronisation inside): chunked initial compression with on-device sketch
// escalation, then nB factorization steps, then one reduction.  The host reads the result
// (loglik, status, ranks) once at the end.
#include "../../include/tlr_b200.h"
#include "tlr_kernels.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return 0;
  return fail(TLR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kLevels = 4;      // sketch widths 16, 32, 64, 128
constexpr int kMaxK = 128;
constexpr int kPowerPasses = 4;       // Z = T^T T P passes per level (FP64 parity path)
constexpr int kPowerPassesMixed = 3;  // mixed path: the exact residual still bounds every tail
// accepted rank must leave `margin` of the k sketch directions unresolved: 12 in the FP64 parity
// path (with 8, an ill-conditioned field, N = 20,000 at range 0.1 and nugget 0.005, kept the
// reference's ranks but missed its log-likelihood by 1.2e-9 relative; with 12 every N = 20,000
// sweep case is within 5e-12), 8 in the mixed path, whose budget is 1e-2 nats
constexpr int kMargin = 12;
constexpr int kMarginMixed = 8;

}  // namespace

namespace tlr {
// lets other translation units of the library report through tlr_last_error()
int set_error(int code, const char* msg) { return fail(code, msg); }
}  // namespace tlr

struct tlr_plan {
  int n = 0, b = 0, nB = 0, ntiles = 0, cap = 0, device = 0;
  cudaStream_t stream = nullptr;
  bool has_data = false;
  // data
  double *xy = nullptr, *y = nullptr, *rhs = nullptr, *z = nullptr;
  // factor
  double *D = nullptr, *U = nullptr, *V = nullptr, *Wd = nullptr, *Yd = nullptr;
  int *rank = nullptr, *rank0 = nullptr, *ti = nullptr, *tj = nullptr;
  // compression chunk
  int chunk = 0, nblk = 0;
  int* need = nullptr;
  double *T = nullptr, *P = nullptr, *Z = nullptr, *C = nullptr, *gscr = nullptr, *gsv = nullptr;
  double *parts = nullptr, *fparts = nullptr;
  // recompression scratch
  int nslots = 0, nsm = 148;
  size_t slot_doubles = 0;
  double* rcs = nullptr;
  int* rc_next = nullptr;  // per factorization step: claims of trailing pairs past the grid
  // look-ahead: POTRF(k+1) runs on a second stream while step k's recompression runs
  cudaStream_t side = nullptr;
  cudaEvent_t ev_panel = nullptr, ev_diag = nullptr;
  // backward: the TLR solve for alpha runs on the side stream, one event per block row
  std::vector<cudaEvent_t> ev_alpha;
  // results
  double *ldpart = nullptr, *qpart = nullptr, *out = nullptr;
  int* status = nullptr;
  // host copies; results land in pinned memory so that evaluations can be queued back to back
  std::vector<int> h_ti, h_tj;
  int *h_rank = nullptr, *h_rank0 = nullptr;  // pinned, ntiles each
  struct HostBlock {
    int status;
    int pad;
    double out[4];
    double grad[3];
    double work[2 * TLR_NKINDS];
  }* hb = nullptr;  // pinned
  double bw_sigma2 = 0.0, bw_inv_range = 0.0, bw_eta = 0.0;
  bool factor_ok = false;  // the last evaluation completed: D, U, V, rank hold its factor
  std::vector<void*> allocs;
  int precision = TLR_PRECISION_FP64;
  // rank map (tlr_plan_rank_map): ntiles initial ranks, then per step k the ranks of its trailing
  // pairs from rlog_off[k]
  int* rlog = nullptr;
  int* blog = nullptr;  // storage bits of every rounding (rule 'mixed'): rlog's layout, then the panel solves'
  int rmode = 0;
  // per initial tile: truncation error ||T - T_r||_F and ||T||_F (the assembled rule's outputs)
  double *tail0 = nullptr, *fro0 = nullptr;
  // storage rule 'mixed': bits of every stored factor tile (index i (i - 1) / 2 + k), and whether the
  // last evaluation used the rule
  int* prec = nullptr;
  int round_store = 0;
  std::vector<size_t> rlog_off;
  // launch accounting and optional per-kernel event timing
  bool prof = false;
  int nu5 = 0;  // covariance: 0 Matern 3/2, 1 Matern 5/2
  int prof_kind = -1;  // -1: every kind
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<int> ev_kind;
  double kms[TLR_NKINDS] = {0};
  long long klaunch[TLR_NKINDS] = {0};
  double kflops[TLR_NKINDS] = {0};
  double kbytes[TLR_NKINDS] = {0};
  // backward pass: one arena sized from the ranks of the evaluation (grown on demand) and the
  // job tables of the selected inversion
  double* bw = nullptr;
  size_t bw_doubles = 0;
  tlr::GemmJob* d_jobs = nullptr;
  size_t d_jobs_cap = 0;
  double** d_ccol = nullptr;
  size_t d_ccol_cap = 0;
  tlr::CopyJob* d_copy = nullptr;
  size_t d_copy_cap = 0;
  // mixed precision: the GEMM operands split to TF32 blocks (one launch at a time) and their tables
  float* tc_area = nullptr;
  size_t tc_area_cap = 0;
  tlr::SplitJob* d_split = nullptr;
  size_t d_split_cap = 0;
  tlr::TcOperands* d_tcops = nullptr;
  size_t d_tcops_cap = 0;
  // forward pass (compression, factorization, solve) captured once per precision in a CUDA graph
  // on a private stream and replayed on `stream`; the launch sequence depends only on the plan
  bool use_graphs = true;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t fwd_exec[2] = {nullptr, nullptr};
  long long fwd_launch[2][TLR_NKINDS] = {};
  // block-row cyclic partition (tlr_plan_set_partition): this plan holds block rows i with
  // i % pworld == prank; tmap lists their tiles (nown of them) for the compression
  int prank = 0, pworld = 1;
  int* tmap = nullptr;
  int nown = 0;
};

namespace {

template <class T>
int dalloc(tlr_plan* p, T** ptr, size_t count) {
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(TLR_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                                   " bytes failed: " + cudaGetErrorString(e));
  }
  p->allocs.push_back(q);
  *ptr = static_cast<T*>(q);
  return 0;
}

void free_all(tlr_plan* p) {
  for (void* q : p->allocs) cudaFree(q);
  p->allocs.clear();
  if (p->bw) cudaFree(p->bw);
  if (p->d_jobs) cudaFree(p->d_jobs);
  if (p->d_ccol) cudaFree(p->d_ccol);
  if (p->d_copy) cudaFree(p->d_copy);
  if (p->tc_area) cudaFree(p->tc_area);
  if (p->d_split) cudaFree(p->d_split);
  if (p->d_tcops) cudaFree(p->d_tcops);
  p->tc_area = nullptr;
  p->d_split = nullptr;
  p->d_tcops = nullptr;
  p->bw = nullptr;
  p->d_jobs = nullptr;
  p->d_ccol = nullptr;
  p->d_copy = nullptr;
}

#define TRY(x)                      \
  do {                              \
    const int _rc = (x);            \
    if (_rc != 0) return _rc;       \
  } while (0)

cudaEvent_t next_event(tlr_plan* p) {
  if (p->ev_used == p->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    p->ev_pool.push_back(e);
  }
  return p->ev_pool[p->ev_used++];
}

// launch one kernel of kind `kind` on stream `st`; with profiling on, bracket it by two events
#define LAUNCH_ON(st, kind, x)                                                      \
  do {                                                                              \
    const bool _ev = p->prof && (p->prof_kind < 0 || p->prof_kind == (kind));      \
    if (_ev) {                                                                      \
      cudaEventRecord(next_event(p), st);                                           \
      p->ev_kind.push_back(kind);                                                   \
    }                                                                               \
    const int _rc = (x);                                                            \
    if (_ev) cudaEventRecord(next_event(p), st);                                    \
    p->klaunch[kind] += 1;                                                          \
    if (_rc != 0) return fail(TLR_ERR_CUDA, std::string("kernel launch failed: ") + \
                                                cudaGetErrorString((cudaError_t)_rc)); \
  } while (0)
#define LAUNCH(kind, x) LAUNCH_ON(p->stream, kind, x)

// The kernels read theta, the rule and the thresholds from the EvalParams of the control block.
int run_compression(tlr_plan* p) {
  cudaStream_t s = p->stream;
  const int ldp = kMaxK;
  const int count = p->pworld > 1 ? p->nown : p->ntiles;  // the tiles this plan compresses
  for (int base = 0; base < count; base += p->chunk) {
    const int nc = std::min(p->chunk, count - base);
    LAUNCH(TLR_K_FILL, tlr::launch_fill_int(p->need, 1, nc, s));
    LAUNCH(TLR_K_GEN, tlr::launch_gen_offdiag(p->xy, p->n, p->b, base, p->ti, p->tj, p->T, nc, p->status, s));
    for (int lev = 0; lev < kLevels; ++lev) {
      const int k = 16 << lev;
      double* Pp = p->P;
      double* Zp = p->Z;
      const int passes = p->precision == TLR_PRECISION_MIXED ? kPowerPassesMixed : kPowerPasses;
      for (int it = 0; it < passes; ++it) {
        LAUNCH(TLR_K_SKETCH, tlr::launch_sketch(p->T, p->n, p->b, k, base, p->ti, p->tj, p->need, Pp, Zp, ldp, it == 0 ? 1 : 0, 0,
                                nc, p->status, s));
        LAUNCH(TLR_K_ORTH, tlr::launch_orth(Zp, p->n, p->b, k, ldp, base, p->tj, p->need, p->gscr, nc, p->status, s));
        std::swap(Pp, Zp);
      }
      const bool fused = tlr::project_resid_fused(p->b, k);  // residual inside the projection pass
      if (fused) {
        LAUNCH(TLR_K_PROJECT, tlr::launch_project_resid(p->T, p->n, p->b, base, p->ti, p->tj, p->need, Pp, p->C, ldp,
                                                        p->parts, p->fparts, nc, p->status, s));
      } else {
        LAUNCH(TLR_K_PROJECT, tlr::launch_sketch(p->T, p->n, p->b, k, base, p->ti, p->tj, p->need, Pp, p->C, ldp, 0, 1, nc,
                                                 p->status, s));
        LAUNCH(TLR_K_RESID, tlr::launch_resid(p->T, p->n, p->b, k, ldp, base, p->ti, p->tj, p->need, Pp, p->C, p->parts,
                                              p->fparts, p->nblk, nc, p->status, s));
      }
      LAUNCH(TLR_K_FINALIZE, tlr::launch_finalize(p->n, p->b, k, ldp, p->cap,
                                p->precision == TLR_PRECISION_MIXED ? kMarginMixed : kMargin, base, p->ti, p->tj,
                                p->need, Pp, p->C, p->parts, p->fparts, fused ? 1 : p->nblk, p->gscr, p->gsv, p->U, p->V,
                                p->rank, lev == kLevels - 1 ? 1 : 0, nc, p->rlog, p->tail0, p->fro0, p->blog, p->status,
                                s));
    }
  }
  return 0;
}

int run_factorization(tlr_plan* p) {
  cudaStream_t s = p->stream, sd = p->side;
  TRY(cuda_check(cudaMemsetAsync(p->rc_next, 0, sizeof(int) * p->nB, s), "pair counters"));
  LAUNCH(TLR_K_DIAG, tlr::launch_diag_build(p->xy, p->n, p->b, 0, p->U, p->Yd, p->rank, p->cap, p->D, p->status, s));
  LAUNCH(TLR_K_POTRF, tlr::launch_potrf(p->D, p->n, p->b, 0, p->rhs, p->z, p->ldpart, p->qpart, p->status, s));
  for (int k = 0; k < p->nB; ++k) {
    LAUNCH(TLR_K_TRSM, tlr::launch_trsm(p->D, p->n, p->b, k, p->nB, p->U, p->V, p->Wd, p->Yd, p->rank, p->cap, p->z, p->rhs,
                                        p->prec, p->blog + p->rlog_off[p->nB], 0, 1, p->status, s));
    const bool ahead = k + 1 < p->nB;
    if (ahead) {
      // A_{k+1,k+1} needs only the panels m <= k, all final once the panel solve of step k is
      // done; step k's recompression touches tiles (i, j) with j > k + 1 only.
      TRY(cuda_check(cudaEventRecord(p->ev_panel, s), "event"));
      TRY(cuda_check(cudaStreamWaitEvent(sd, p->ev_panel, 0), "wait"));
      LAUNCH_ON(sd, TLR_K_DIAG, tlr::launch_diag_build(p->xy, p->n, p->b, k + 1, p->U, p->Yd, p->rank, p->cap,
                                                       p->D, p->status, sd));
      LAUNCH_ON(sd, TLR_K_POTRF, tlr::launch_potrf(p->D, p->n, p->b, k + 1, p->rhs, p->z, p->ldpart, p->qpart,
                                                   p->status, sd));
      TRY(cuda_check(cudaEventRecord(p->ev_diag, sd), "event"));
    }
    LAUNCH(TLR_K_RECOMPRESS, tlr::launch_recompress(p->n, p->b, k, p->nB, p->U, p->V, p->rank, p->cap, p->rcs,
                                                    p->slot_doubles, p->nslots, p->rc_next + k,
                                                    p->rlog + p->rlog_off[k], p->blog + p->rlog_off[k], 0, 1,
                                                    p->status, s));
    if (ahead) TRY(cuda_check(cudaStreamWaitEvent(s, p->ev_diag, 0), "wait"));
  }
  LAUNCH(TLR_K_FINISH, tlr::launch_finish(p->nB, p->n, p->ldpart, p->qpart, p->out, p->status, s));
  return 0;
}

// The forward pass after launch_set_params: ranks cleared, right-hand side, compression (the
// initial ranks kept in rank0), factorization with the fused forward solve.
int forward_sequence(tlr_plan* p) {
  cudaStream_t s = p->stream;
  TRY(cuda_check(cudaMemsetAsync(p->rank, 0, sizeof(int) * std::max(p->ntiles, 1), s), "reset ranks"));
  TRY(cuda_check(cudaMemcpyAsync(p->rhs, p->y, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, s), "rhs"));
  TRY(run_compression(p));
  if (p->ntiles > 0)
    TRY(cuda_check(cudaMemcpyAsync(p->rank0, p->rank, sizeof(int) * p->ntiles, cudaMemcpyDeviceToDevice, s),
                   "rank0"));
  TRY(run_factorization(p));
  return 0;
}

// Capture forward_sequence on the plan's private stream (nothing runs) and instantiate it.  The
// launches counted during the capture become the graph's per-replay counts.
int capture_forward(tlr_plan* p, int g) {
  if (!p->cap_stream)
    TRY(cuda_check(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking), "capture stream"));
  long long before[TLR_NKINDS];
  std::memcpy(before, p->klaunch, sizeof(before));
  cudaStream_t user = p->stream;
  p->stream = p->cap_stream;
  int rc = cuda_check(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeRelaxed), "begin capture");
  if (!rc) {
    rc = forward_sequence(p);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(p->cap_stream, &graph);
    if (!rc && e != cudaSuccess) rc = cuda_check(e, "end capture");
    if (!rc) rc = cuda_check(cudaGraphInstantiate(&p->fwd_exec[g], graph, 0), "instantiate forward graph");
    if (graph) cudaGraphDestroy(graph);
  }
  p->stream = user;
  for (int i = 0; i < TLR_NKINDS; ++i) {
    p->fwd_launch[g][i] = p->klaunch[i] - before[i];
    p->klaunch[i] = before[i];
  }
  if (rc) {
    cudaGetLastError();
    p->fwd_exec[g] = nullptr;
  }
  return rc;
}

// One forward pass on the plan's stream: the captured graph of the plan's precision (captured on
// first use), or the launches themselves while per-kernel event timing is on or graphs are off.
int run_forward(tlr_plan* p) {
  if (!p->use_graphs || p->prof) return forward_sequence(p);
  const int g = p->precision == TLR_PRECISION_MIXED ? 1 : 0;
  if (!p->fwd_exec[g]) TRY(capture_forward(p, g));
  TRY(cuda_check(cudaGraphLaunch(p->fwd_exec[g], p->stream), "forward graph launch"));
  for (int i = 0; i < TLR_NKINDS; ++i) p->klaunch[i] += p->fwd_launch[g][i];
  return 0;
}

// The evaluation's parameters (thresholds: codes/17_tlr_cholesky_pilot.py:143-150 and
// codes/11_tlr_rank_rules.py:81-98, emax = tau b m_theta / N with b the largest tile).
tlr::EvalParams make_params(const tlr_plan* p, const double theta[3], int rule, double value) {
  tlr::EvalParams prm{};
  const double sigma2 = theta[0], range = theta[1], eta = theta[2];
  prm.sigma2 = sigma2;
  prm.inv_range = 1.0 / range;
  prm.nugget = sigma2 * eta;
  prm.rule_fixed = rule == TLR_RULE_FIXED ? 1 : 0;
  prm.thr_rel = prm.rule_fixed ? value : 0.0;
  prm.thr_abs = prm.rule_fixed ? 0.0 : value * (double)std::min(p->b, p->n) * sigma2 * eta / (double)p->n;
  prm.rmode = p->rmode;
  prm.round_store = rule == TLR_RULE_MIXED ? 1 : 0;
  prm.nu5 = p->nu5;
  prm.tmap = p->pworld > 1 ? p->tmap : nullptr;
  return prm;
}

}  // namespace


// ------------------------------------------------------------------------------------------
// Backward pass (gradient).  See csrc/tlr_backward.cu for the recurrence.
namespace {

template <class T>
int grow(T** ptr, size_t* cap, size_t need) {
  if (need <= *cap && *ptr) return 0;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *cap = 0;
  const size_t want = std::max<size_t>(need, 1) + need / 4;
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, want * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(TLR_ERR_NOMEM, std::string("backward arena: ") + cudaGetErrorString(e));
  }
  *ptr = static_cast<T*>(q);
  *cap = want;
  return 0;
}

// Split tables of one launch of the tensor-core GEMM: every distinct operand (pointer, leading
// dimension, layout, rows, K) of the jobs once, at float offsets of a scratch area (the SplitJob's
// dst stays NULL until the area is known); per job the offsets of its op(A) and op(B)^T blocks,
// SIZE_MAX for a job without products.
struct TcSplitPlan {
  std::vector<tlr::SplitJob> splits;
  std::vector<size_t> split_off;
  std::vector<std::pair<size_t, size_t>> job_off;
  int max_blocks = 0;
  size_t floats = 0;
};

static void tc_split_plan(const tlr::GemmJob* jobs, int count, TcSplitPlan& out) {
  std::map<std::tuple<const double*, int, int, int, int>, size_t> seen;
  auto panel = [&](const double* src, int ld, int kcont, int rows, int K) {
    const auto key = std::make_tuple(src, ld, kcont, rows, K);
    const auto it = seen.find(key);
    if (it != seen.end()) return it->second;
    const size_t off = out.floats;
    out.splits.push_back({src, nullptr, ld, kcont, rows, K});
    out.split_off.push_back(off);
    out.max_blocks = std::max(out.max_blocks, tlr::tc_panel_blocks(rows, K));
    out.floats += tlr::tc_panel_floats(rows, K);
    seen.emplace(key, off);
    return off;
  };
  for (int q = 0; q < count; ++q) {
    const tlr::GemmJob& j = jobs[q];
    if (j.M > 0 && j.N > 0 && j.K > 0)
      out.job_off.push_back({panel(j.A, j.lda, j.transA ? 1 : 0, j.M, j.K), panel(j.B, j.ldb, j.transB ? 0 : 1, j.N, j.K)});
    else
      out.job_off.push_back({SIZE_MAX, SIZE_MAX});
  }
}

struct LaunchRange {
  int kind;      // 0 gemm, 1 copy, 2 alpha, 3 dtrace, 4 gemm that stays FP64 in mixed mode
  size_t first;  // index of the first job
  int count;
  int max_m, max_n;
  int m;
  size_t part_off;
};

// Queue the backward pass of the last successful forward evaluation on the plan's stream (the
// ranks of that evaluation are in the pinned host copy); the gradient lands in the pinned block.
int run_backward(tlr_plan* p, double sigma2, double inv_range, double eta) {
  const int nB = p->nB, b = p->b, n = p->n;
  const size_t B = (size_t)b, BB = B * B;
  auto bsz = [&](int i) { return std::min(b, n - i * b); };
  auto r = [&](int i, int m) { return p->h_rank[(size_t)i * (i - 1) / 2 + m]; };
  // layout from the ranks
  std::vector<std::vector<int>> offU(nB), offV(nB);
  std::vector<int> Rlt(nB), Rcol(nB);
  for (int i = 0; i < nB; ++i) {
    offU[i].assign(i + 1, 0);
    for (int m = 0; m < i; ++m) offU[i][m + 1] = offU[i][m] + r(i, m);
    Rlt[i] = offU[i][i];
  }
  for (int m = 0; m < nB; ++m) {
    offV[m].assign(nB + 1, 0);
    for (int j = m + 1; j < nB; ++j) offV[m][j + 1] = offV[m][j] + r(j, m);
    Rcol[m] = offV[m][nB];
  }
  size_t o = 0;
  const size_t oLi = o; o += (size_t)nB * BB;
  const size_t oZ = o; o += (size_t)nB * BB;
  std::vector<size_t> oUcat(nB);
  for (int i = 0; i < nB; ++i) { oUcat[i] = o; o += B * Rlt[i]; }
  std::vector<std::vector<size_t>> oC(nB);
  for (int i = 0; i < nB; ++i) {
    oC[i].assign(i + 1, 0);
    for (int m = 0; m <= i; ++m) { oC[i][m] = o; o += B * Rcol[m]; }
  }
  int Rmax = 1;
  for (int m = 0; m < nB; ++m) Rmax = std::max(Rmax, Rcol[m]);
  const size_t oVs = o; o += B * Rmax;
  const size_t oVp = o; o += B * Rmax;
  const size_t oAl = o; o += (size_t)nB * B;
  const size_t oWk = o; o += B + (size_t)std::max(Rmax, 1);
  const int nb32 = (b + 31) / 32;
  std::vector<size_t> part_off(nB);
  size_t nparts = 0;
  for (int m = 0; m < nB; ++m) { part_off[m] = nparts; nparts += (size_t)(nB - m) * nb32 * nb32; }
  const size_t oPart = o; o += 3 * nparts;
  const size_t oGrad = o; o += 4;
  TRY(grow(&p->bw, &p->bw_doubles, o));
  double* base = p->bw;
  double* Li = base + oLi;
  double* Zb = base + oZ;
  double* Vs = base + oVs;
  double* Vp = base + oVp;
  auto Cp = [&](int i, int m) { return base + oC[i][m]; };
  auto Ucat = [&](int i) { return base + oUcat[i]; };
  auto Ut = [&](int i, int m) { return p->U + ((size_t)i * (i - 1) / 2 + m) * B * p->cap; };
  auto Vt = [&](int i, int m) { return p->V + ((size_t)i * (i - 1) / 2 + m) * B * p->cap; };

  std::vector<tlr::GemmJob> jobs;
  std::vector<double*> ccol;
  std::vector<size_t> ccol_first;  // per job: index into ccol, or SIZE_MAX
  std::vector<tlr::CopyJob> copies;
  std::vector<LaunchRange> plan;
  auto gemm = [&](const double* A, int lda, int tA, const double* Bm, int ldb, int tB, double* C, int ldc, int M,
                  int N, int K, double alpha, double beta) {
    tlr::GemmJob j{A, Bm, C, nullptr, lda, ldb, ldc, M, N, K, tA, tB, alpha, beta};
    jobs.push_back(j);
    ccol_first.push_back(SIZE_MAX);
  };
  auto begin_gemm = [&](int m) { plan.push_back({0, jobs.size(), 0, 0, 0, m, 0}); };
  auto end_gemm = [&]() {
    LaunchRange& L = plan.back();
    L.count = (int)(jobs.size() - L.first);
    for (size_t q = L.first; q < jobs.size(); ++q) {
      L.max_m = std::max(L.max_m, jobs[q].M);
      L.max_n = std::max(L.max_n, jobs[q].N);
    }
    if (L.count == 0 || L.max_m == 0 || L.max_n == 0) plan.pop_back();
  };
  // gather every row's U factors once: Ucat_i = [U_i0 ... U_i,i-1]
  plan.push_back({1, copies.size(), 0, 0, 0, -1, 0});
  for (int i = 0; i < nB; ++i)
    for (int m = 0; m < i; ++m)
      if (r(i, m)) copies.push_back({Ut(i, m), Ucat(i) + (size_t)offU[i][m] * B, b, b, bsz(i), r(i, m)});
  plan.back().count = (int)(copies.size() - plan.back().first);
  for (int m = nB - 1; m >= 0; --m) {
    const int bm = bsz(m);
    // Vstack_m = [V_jm]_{j>m}
    plan.push_back({1, copies.size(), 0, 0, 0, m, 0});
    for (int j = m + 1; j < nB; ++j)
      if (r(j, m)) copies.push_back({Vt(j, m), Vs + (size_t)offV[m][j] * B, b, b, bm, r(j, m)});
    plan.back().count = (int)(copies.size() - plan.back().first);
    // Vp_m = Li_m^T Vstack_m ; Z_mm = Li_m^T Li_m (the diagonal blocks carry tr(Z), which nearly
    // cancels against alpha^T alpha: they stay FP64 in the mixed path)
    begin_gemm(m);
    if (Rcol[m]) gemm(Li + (size_t)m * BB, b, 1, Vs, b, 0, Vp, b, bm, Rcol[m], bm, 1.0, 0.0);
    end_gemm();
    begin_gemm(m);
    gemm(Li + (size_t)m * BB, b, 1, Li + (size_t)m * BB, b, 0, Zb, b, bm, bm, bm, 1.0, 0.0);
    end_gemm();
    if (!plan.empty() && plan.back().kind == 0 && plan.back().m == m) plan.back().kind = 4;
    // Z_im = -C_im Vp_m^T, i > m
    begin_gemm(m);
    for (int i = m + 1; i < nB; ++i)
      gemm(Cp(i, m), b, 0, Vp, b, 1, Zb + (size_t)(i - m) * BB, b, bsz(i), bm, Rcol[m], -1.0, 0.0);
    end_gemm();
    // products of Z_im (i > m) with the U panels, scattered into the C buffers
    begin_gemm(m);
    for (int i = m + 1; i < nB; ++i) {
      const double* Zim = Zb + (size_t)(i - m) * BB;
      const int Nt = offU[i][m + 1];  // PBT_im = Z_im^T [U_i0 .. U_im]
      if (Nt) {
        gemm(Zim, b, 1, Ucat(i), b, 0, nullptr, b, bm, Nt, bsz(i), 1.0, 0.0);
        ccol_first.back() = ccol.size();
        for (int mp = 0; mp <= m; ++mp)
          for (int c = 0; c < r(i, mp); ++c) ccol.push_back(Cp(m, mp) + (size_t)(offV[mp][i] + c) * B);
      }
      if (m >= 1 && Rlt[m]) {  // PB_im = Z_im [U_m0 .. U_m,m-1]
        gemm(Zim, b, 0, Ucat(m), b, 0, nullptr, b, bsz(i), Rlt[m], bm, 1.0, 0.0);
        ccol_first.back() = ccol.size();
        for (int mp = 0; mp < m; ++mp)
          for (int c = 0; c < r(m, mp); ++c) ccol.push_back(Cp(i, mp) + (size_t)(offV[mp][m] + c) * B);
      }
    }
    end_gemm();
    // Z_mm -= C_mm Vp_m^T (FP64 in both paths)
    begin_gemm(m);
    if (Rcol[m]) gemm(Cp(m, m), b, 0, Vp, b, 1, Zb, b, bm, bm, Rcol[m], -1.0, 1.0);
    end_gemm();
    if (Rcol[m] && !plan.empty() && plan.back().kind == 0 && plan.back().m == m) plan.back().kind = 4;
    // PB_mm = Z_mm [U_m0 .. U_m,m-1]
    begin_gemm(m);
    if (m >= 1 && Rlt[m]) {
      gemm(Zb, b, 0, Ucat(m), b, 0, nullptr, b, bm, Rlt[m], bm, 1.0, 0.0);
      ccol_first.back() = ccol.size();
      for (int mp = 0; mp < m; ++mp)
        for (int c = 0; c < r(m, mp); ++c) ccol.push_back(Cp(m, mp) + (size_t)(offV[mp][m] + c) * B);
    }
    end_gemm();
    plan.push_back({2, 0, 1, 0, 0, m, 0});
    plan.push_back({3, 0, 1, 0, 0, m, part_off[m]});
  }
  // upload the tables
  TRY(grow(&p->d_jobs, &p->d_jobs_cap, jobs.size()));
  TRY(grow(&p->d_ccol, &p->d_ccol_cap, ccol.size()));
  TRY(grow(&p->d_copy, &p->d_copy_cap, copies.size()));
  for (size_t q = 0; q < jobs.size(); ++q)
    if (ccol_first[q] != SIZE_MAX) jobs[q].ccol = p->d_ccol + ccol_first[q];
  cudaStream_t s = p->stream;
  if (!jobs.empty())
    TRY(cuda_check(cudaMemcpyAsync(p->d_jobs, jobs.data(), jobs.size() * sizeof(tlr::GemmJob), cudaMemcpyHostToDevice, s),
                   "jobs"));
  if (!ccol.empty())
    TRY(cuda_check(cudaMemcpyAsync(p->d_ccol, ccol.data(), ccol.size() * sizeof(double*), cudaMemcpyHostToDevice, s),
                   "ccol"));
  if (!copies.empty())
    TRY(cuda_check(cudaMemcpyAsync(p->d_copy, copies.data(), copies.size() * sizeof(tlr::CopyJob),
                                   cudaMemcpyHostToDevice, s),
                   "copies"));
  // mixed precision: split tables of every tensor-core GEMM launch; the launches share one area
  // (each split runs right before its GEMM on the same stream)
  std::vector<size_t> split_first(plan.size(), 0);
  std::vector<int> split_count(plan.size(), 0), split_blocks(plan.size(), 0);
  if (p->precision == TLR_PRECISION_MIXED) {
    std::vector<tlr::SplitJob> splits;
    std::vector<size_t> soff;
    std::vector<std::pair<size_t, size_t>> joff(jobs.size(), {SIZE_MAX, SIZE_MAX});
    size_t area = 0;
    for (size_t li = 0; li < plan.size(); ++li) {
      const LaunchRange& L = plan[li];
      if (L.kind != 0 || L.count == 0) continue;
      TcSplitPlan sp;
      tc_split_plan(jobs.data() + L.first, L.count, sp);
      split_first[li] = splits.size();
      split_count[li] = (int)sp.splits.size();
      split_blocks[li] = sp.max_blocks;
      splits.insert(splits.end(), sp.splits.begin(), sp.splits.end());
      soff.insert(soff.end(), sp.split_off.begin(), sp.split_off.end());
      for (int q = 0; q < L.count; ++q) joff[L.first + q] = sp.job_off[q];
      area = std::max(area, sp.floats);
    }
    TRY(grow(&p->tc_area, &p->tc_area_cap, area));
    TRY(grow(&p->d_split, &p->d_split_cap, splits.size()));
    TRY(grow(&p->d_tcops, &p->d_tcops_cap, jobs.size()));
    for (size_t q = 0; q < splits.size(); ++q) splits[q].dst = p->tc_area + soff[q];
    std::vector<tlr::TcOperands> ops(jobs.size(), {nullptr, nullptr});
    for (size_t q = 0; q < jobs.size(); ++q)
      if (joff[q].first != SIZE_MAX) ops[q] = {p->tc_area + joff[q].first, p->tc_area + joff[q].second};
    if (!splits.empty())
      TRY(cuda_check(cudaMemcpyAsync(p->d_split, splits.data(), splits.size() * sizeof(tlr::SplitJob),
                                     cudaMemcpyHostToDevice, s),
                     "split table"));
    if (!ops.empty())
      TRY(cuda_check(cudaMemcpyAsync(p->d_tcops, ops.data(), ops.size() * sizeof(tlr::TcOperands),
                                     cudaMemcpyHostToDevice, s),
                     "operand table"));
  }
  // launches
  LAUNCH(TLR_K_TRI_INV, tlr::launch_tri_inv(p->D, Li, n, b, nB, p->status, s));
  // alpha = Sigma_t^{-1} y (block rows nB-1 .. 0) needs only the factor, z and the inverses of
  // the diagonal tiles: it runs on the side stream while the selected-inversion GEMMs run here
  while ((int)p->ev_alpha.size() < nB) {
    cudaEvent_t e;
    TRY(cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event"));
    p->ev_alpha.push_back(e);
  }
  TRY(cuda_check(cudaEventRecord(p->ev_panel, s), "event"));
  TRY(cuda_check(cudaStreamWaitEvent(p->side, p->ev_panel, 0), "wait"));
  for (int m = nB - 1; m >= 0; --m) {
    LAUNCH_ON(p->side, TLR_K_ALPHA, tlr::launch_alpha_step(n, b, m, nB, p->U, p->V, p->rank, p->cap, Li, p->z,
                                                           base + oAl, base + oWk, p->status, p->side));
    TRY(cuda_check(cudaEventRecord(p->ev_alpha[m], p->side), "event"));
  }
  for (size_t li = 0; li < plan.size(); ++li) {
    const LaunchRange& L = plan[li];
    if (L.kind == 4) {
      LAUNCH(TLR_K_BWD_GEMM, tlr::launch_dgemm_batched(p->d_jobs + L.first, L.count, L.max_m, L.max_n, p->status,
                                                        TLR_K_BWD_GEMM, s));
    } else if (L.kind == 0) {
      if (p->precision == TLR_PRECISION_MIXED) {
        if (split_count[li])
          LAUNCH(TLR_K_BWD_GEMM, tlr::launch_split_tf32(p->d_split + split_first[li], split_count[li],
                                                         split_blocks[li], p->status, TLR_K_BWD_GEMM, s));
        LAUNCH(TLR_K_BWD_GEMM, tlr::launch_gemm_tc3(p->d_jobs + L.first, p->d_tcops + L.first, L.count, L.max_m,
                                                     L.max_n, p->status, TLR_K_BWD_GEMM, s));
      }
      else
        LAUNCH(TLR_K_BWD_GEMM, tlr::launch_dgemm_batched(p->d_jobs + L.first, L.count, L.max_m, L.max_n, p->status,
                                                          TLR_K_BWD_GEMM, s));
    } else if (L.kind == 1) {
      if (L.count) LAUNCH(TLR_K_BWD_COPY, tlr::launch_copy_cols(p->d_copy + L.first, L.count, p->status, s));
    } else if (L.kind == 2) {
      TRY(cuda_check(cudaStreamWaitEvent(s, p->ev_alpha[L.m], 0), "wait"));
    } else {
      LAUNCH(TLR_K_DTRACE, tlr::launch_dtrace_step(p->xy, n, b, L.m, nB, sigma2, inv_range, p->nu5, eta, Zb, base + oAl,
                                                   base + oPart + 3 * L.part_off, p->status, s));
    }
  }
  LAUNCH(TLR_K_GRAD_FINISH, tlr::launch_grad_finish(base + oPart, (long)nparts, base + oGrad, p->status, s));
  TRY(cuda_check(cudaMemcpyAsync(p->hb->grad, base + oGrad, sizeof(double) * 3, cudaMemcpyDeviceToHost, s), "grad"));
  TRY(cuda_check(cudaMemcpyAsync(&p->hb->status, p->status, sizeof(int), cudaMemcpyDeviceToHost, s), "status"));
  TRY(cuda_check(cudaMemcpyAsync(p->hb->work, p->status + 4, sizeof(double) * 2 * TLR_NKINDS,
                                 cudaMemcpyDeviceToHost, s),
                 "work"));
  return 0;
}

// Wait for the backward pass queued by run_backward and collect its gradient.
int finish_backward(tlr_plan* p, double* grad_host) {
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  TRY(cuda_check(cudaStreamSynchronize(p->stream), "backward"));
  const int status = p->hb->status;
  const double* work = p->hb->work;
  if (p->prof) {
    for (size_t q = 0; q < p->ev_kind.size(); ++q) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p->ev_pool[2 * q], p->ev_pool[2 * q + 1]);
      p->kms[p->ev_kind[q]] += ms;
    }
  }
  p->ev_used = 0;
  p->ev_kind.clear();
  for (int q = TLR_K_BWD_GEMM; q < TLR_NKINDS; ++q) {  // the forward's counts were taken already
    p->kflops[q] += work[2 * q];
    p->kbytes[q] += work[2 * q + 1];
  }
  if (status != 0) return fail(status < 0 ? status : TLR_ERR_CUDA, "backward pass failed");
  for (int a = 0; a < 3; ++a) grad_host[a] = p->hb->grad[a];
  return 0;
}

}  // namespace

extern "C" {

const char* tlr_last_error(void) { return g_err.c_str(); }

int tlr_plan_create(tlr_plan** plan, int n, int b, int cap, int device, void* stream) {
  if (!plan) return fail(TLR_ERR_ARG, "plan is NULL");
  *plan = nullptr;
  if (n < 1 || b < 1) return fail(TLR_ERR_ARG, "n and b must be positive");
  if (b > 1024) return fail(TLR_ERR_ARG, "tile size b must be <= 1024");
  if ((n + b - 1) / b > 1024) return fail(TLR_ERR_ARG, "at most 1024 tiles per side (N / b <= 1024)");
  if (cap < 1 || cap > 128) return fail(TLR_ERR_ARG, "rank capacity must be in [1, 128]");
  TRY(cuda_check(cudaSetDevice(device), "cudaSetDevice"));
  tlr_plan* p = new tlr_plan();
  p->n = n;
  p->b = b;
  p->nB = (n + b - 1) / b;
  p->ntiles = p->nB * (p->nB - 1) / 2;
  p->cap = cap;
  p->device = device;
  p->stream = static_cast<cudaStream_t>(stream);
  const size_t N = (size_t)n, B = (size_t)b;
  int rc = 0;
  auto A = [&](int r) {
    if (rc == 0 && r != 0) rc = r;
  };
  A(dalloc(p, &p->xy, 2 * N));
  A(dalloc(p, &p->y, N));
  A(dalloc(p, &p->rhs, (size_t)p->nB * B));
  A(dalloc(p, &p->z, (size_t)p->nB * B));
  A(dalloc(p, &p->D, (size_t)p->nB * B * B));
  const size_t nt = std::max(p->ntiles, 1);
  A(dalloc(p, &p->U, nt * B * cap));
  A(dalloc(p, &p->V, nt * B * cap));
  A(dalloc(p, &p->Wd, nt * (size_t)cap * cap));
  A(dalloc(p, &p->Yd, nt * B * cap));
  A(dalloc(p, &p->rank, nt));
  A(dalloc(p, &p->rank0, nt));
  A(dalloc(p, &p->ti, nt));
  A(dalloc(p, &p->tj, nt));
  // compression chunk: bounded so T + panels stay within ~4 GB
  const size_t per_tile = (B * B + 4 * B * kMaxK + 2 * (size_t)kMaxK * kMaxK) * 8;
  p->chunk = (int)std::max<size_t>(1, std::min<size_t>(nt, (size_t)4 * 1024 * 1024 * 1024 / per_tile));
  p->nblk = (b + 63) / 64;
  const size_t ch = (size_t)p->chunk;
  A(dalloc(p, &p->need, ch));
  A(dalloc(p, &p->T, ch * B * B));
  A(dalloc(p, &p->P, ch * B * kMaxK));
  A(dalloc(p, &p->Z, ch * B * kMaxK));
  A(dalloc(p, &p->C, ch * B * kMaxK));
  A(dalloc(p, &p->gscr, ch * B * kMaxK));
  A(dalloc(p, &p->gsv, ch * 2 * (size_t)kMaxK * kMaxK));
  A(dalloc(p, &p->parts, ch * p->nblk));
  A(dalloc(p, &p->fparts, ch * p->nblk));
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  p->nsm = nsm;
  p->nslots = nsm * tlr::rc_blocks_per_sm();  // resident recompression CTAs
  p->slot_doubles = tlr::rc_slot_doubles(b, cap);
  A(dalloc(p, &p->rcs, (size_t)p->nslots * p->slot_doubles));
  A(dalloc(p, &p->rc_next, (size_t)p->nB));
  // rank map: the initial ranks, then the trailing pairs of every step
  p->rlog_off.assign((size_t)p->nB + 1, 0);
  size_t rl = nt;
  for (int k = 0; k < p->nB; ++k) {
    p->rlog_off[k] = rl;
    const size_t mB = (size_t)(p->nB - k - 1);
    rl += mB * (mB > 0 ? mB - 1 : 0) / 2;
  }
  p->rlog_off[p->nB] = rl;
  A(dalloc(p, &p->rlog, rl));
  A(dalloc(p, &p->blog, rl + nt));
  A(dalloc(p, &p->tail0, nt));
  A(dalloc(p, &p->fro0, nt));
  A(dalloc(p, &p->prec, nt));
  if (rc == 0) {
    rc = cuda_check(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking), "side stream");
    if (!rc) rc = cuda_check(cudaEventCreateWithFlags(&p->ev_panel, cudaEventDisableTiming), "event");
    if (!rc) rc = cuda_check(cudaEventCreateWithFlags(&p->ev_diag, cudaEventDisableTiming), "event");
  }
  A(dalloc(p, &p->ldpart, (size_t)p->nB));
  A(dalloc(p, &p->qpart, (size_t)p->nB));
  A(dalloc(p, &p->out, 4));
  // control block: status, padding, [flops, bytes] per kernel kind, the evaluation's parameters
  A(dalloc(p, &p->status, (tlr::kControlBytes + sizeof(int) - 1) / sizeof(int)));
  if (rc != 0) {
    free_all(p);
    delete p;
    return rc;
  }
  // tile index tables: t = i (i - 1) / 2 + j
  p->h_ti.resize(nt);
  p->h_tj.resize(nt);
  for (int i = 0; i < p->nB; ++i)
    for (int j = 0; j < i; ++j) {
      const int t = i * (i - 1) / 2 + j;
      p->h_ti[t] = i;
      p->h_tj[t] = j;
    }
  if (p->ntiles > 0) {
    rc = cuda_check(cudaMemcpy(p->ti, p->h_ti.data(), sizeof(int) * p->ntiles, cudaMemcpyHostToDevice), "copy ti");
    if (!rc) rc = cuda_check(cudaMemcpy(p->tj, p->h_tj.data(), sizeof(int) * p->ntiles, cudaMemcpyHostToDevice), "copy tj");
  }
  if (rc != 0) {
    free_all(p);
    delete p;
    return rc;
  }
  void *hr = nullptr, *hr0 = nullptr, *hbk = nullptr;
  rc = cuda_check(cudaMallocHost(&hr, sizeof(int) * nt), "pinned ranks");
  if (!rc) rc = cuda_check(cudaMallocHost(&hr0, sizeof(int) * nt), "pinned ranks");
  if (!rc) rc = cuda_check(cudaMallocHost(&hbk, sizeof(tlr_plan::HostBlock)), "pinned results");
  p->h_rank = static_cast<int*>(hr);
  p->h_rank0 = static_cast<int*>(hr0);
  p->hb = static_cast<tlr_plan::HostBlock*>(hbk);
  if (rc != 0) {
    tlr_plan_destroy(p);
    return rc;
  }
  std::memset(p->h_rank, 0, sizeof(int) * nt);
  std::memset(p->h_rank0, 0, sizeof(int) * nt);
  *plan = p;
  return 0;
}

void tlr_plan_destroy(tlr_plan* plan) {
  if (!plan) return;
  cudaSetDevice(plan->device);
  if (plan->stream) cudaStreamSynchronize(plan->stream);
  for (cudaEvent_t e : plan->ev_pool) cudaEventDestroy(e);
  for (cudaEvent_t e : plan->ev_alpha) cudaEventDestroy(e);
  if (plan->ev_panel) cudaEventDestroy(plan->ev_panel);
  if (plan->ev_diag) cudaEventDestroy(plan->ev_diag);
  if (plan->side) cudaStreamDestroy(plan->side);
  for (cudaGraphExec_t g : plan->fwd_exec)
    if (g) cudaGraphExecDestroy(g);
  if (plan->cap_stream) cudaStreamDestroy(plan->cap_stream);
  if (plan->h_rank) cudaFreeHost(plan->h_rank);
  if (plan->h_rank0) cudaFreeHost(plan->h_rank0);
  if (plan->hb) cudaFreeHost(plan->hb);
  free_all(plan);
  delete plan;
}

int tlr_morton_order(const double* xy_dev, int n, int order, long long* perm_dev, void* stream) {
  if (n < 1 || !xy_dev || !perm_dev) return fail(TLR_ERR_ARG, "invalid arguments to tlr_morton_order");
  if (order < 1 || order > 12) return fail(TLR_ERR_ARG, "order must be in [1, 12]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned* work = nullptr;
  const cudaError_t e = cudaMallocAsync(&work, sizeof(unsigned) * tlr::morton_work_words(n, order), s);
  int rc = 0;
  if (e != cudaSuccess) rc = fail(TLR_ERR_NOMEM, std::string("morton scratch: ") + cudaGetErrorString(e));
  if (!rc) {
    const int lr = tlr::launch_morton(xy_dev, n, order, work, perm_dev, s);
    if (lr) rc = fail(TLR_ERR_CUDA, std::string("morton launch: ") + cudaGetErrorString((cudaError_t)lr));
  }
  if (work) cudaFreeAsync(work, s);
  if (!rc) rc = cuda_check(cudaStreamSynchronize(s), "morton sync");
  return rc;
}

int tlr_set_data(tlr_plan* p, const double* xy_dev, const double* y_dev) {
  if (!p || !xy_dev || !y_dev) return fail(TLR_ERR_ARG, "invalid arguments to tlr_set_data");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  TRY(cuda_check(cudaMemcpyAsync(p->xy, xy_dev, sizeof(double) * 2 * p->n, cudaMemcpyDeviceToDevice, p->stream),
                 "copy sites"));
  TRY(cuda_check(cudaMemcpyAsync(p->y, y_dev, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, p->stream),
                 "copy observations"));
  p->has_data = true;
  return 0;
}

static void fill_info(const tlr_plan* p, int status, const double* out, tlr_info* info, int* factor_ranks,
                      int* sigma_ranks) {
  const int nB = p->nB, b = p->b, n = p->n;
  auto bsz = [&](int i) { return std::min(b, n - i * b); };
  long long stored0 = 0;
  int maxr0 = 0;
  for (int i = 0; i < nB; ++i) {
    stored0 += (long long)bsz(i) * bsz(i);
    for (int j = 0; j < i; ++j) {
      const int r = p->h_rank0[i * (i - 1) / 2 + j];
      stored0 += 2LL * r * std::max(bsz(i), bsz(j));
      maxr0 = std::max(maxr0, r);
    }
  }
  if (sigma_ranks) {
    int q = 0;
    for (int i = 0; i < nB; ++i)
      for (int j = 0; j < i; ++j) sigma_ranks[q++] = p->h_rank0[i * (i - 1) / 2 + j];
  }
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->stored_sigma = stored0;
    info->max_rank_sigma = maxr0;
    info->completed = status == 0 ? 1 : 0;
    info->failed_at = status > 0 ? status - 1 : -1;
  }
  if (status != 0) return;
  long long stored = 0;
  long long rsum = 0;
  int rmax = 0, cnt = 0, q = 0;
  for (int k = 0; k < nB; ++k) stored += (long long)bsz(k) * bsz(k);
  for (int k = 0; k < nB; ++k)
    for (int i = k + 1; i < nB; ++i) {
      const int r = p->h_rank[i * (i - 1) / 2 + k];
      stored += 2LL * r * bsz(i);
      rsum += r;
      rmax = std::max(rmax, r);
      ++cnt;
      if (factor_ranks) factor_ranks[q++] = r;
    }
  if (info) {
    info->stored_factor = stored;
    info->mean_rank_factor = cnt ? (double)rsum / cnt : 0.0;
    info->max_rank_factor = rmax;
    info->logdet = out[1];
    info->quad = out[2];
  }
}

}  // extern "C"

namespace {

// Queue one forward evaluation (compression, factorization, solve) on the plan's stream; the
// status, log-likelihood, work counters and ranks are copied to pinned host memory at the end.
int enqueue_results(tlr_plan* p);

int enqueue_forward(tlr_plan* p, const double theta[3], int rule, double value) {
  if (!p || !theta) return fail(TLR_ERR_ARG, "invalid arguments to tlr_loglik");
  if (!p->has_data) return fail(TLR_ERR_NOT_READY, "tlr_set_data has not been called");
  if (p->pworld > 1) return fail(TLR_ERR_ARG, "the plan is partitioned: evaluate it through the tlr_dist_* steps");
  if (rule != TLR_RULE_FIXED && rule != TLR_RULE_ADAPTIVE && rule != TLR_RULE_MIXED)
    return fail(TLR_ERR_ARG, "rule must be fixed, adaptive or mixed");
  const double sigma2 = theta[0], range = theta[1], eta = theta[2];
  if (!(range > 0.0) || !std::isfinite(sigma2) || !std::isfinite(eta) || !std::isfinite(range))
    return fail(TLR_ERR_ARG, "theta must be finite with range > 0");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  cudaStream_t s = p->stream;
  p->factor_ok = false;
  // rule 'mixed' (17:145-148): the adaptive thresholds, every stored factor pair rounded
  p->round_store = rule == TLR_RULE_MIXED ? 1 : 0;
  LAUNCH(TLR_K_FILL, tlr::launch_set_params(p->status, make_params(p, theta, rule, value), s));
  TRY(run_forward(p));
  TRY(enqueue_results(p));
  p->bw_sigma2 = sigma2;
  p->bw_inv_range = 1.0 / range;
  p->bw_eta = eta;
  return 0;
}

// Copy the status, log-likelihood parts, work counters and ranks to pinned host memory.
int enqueue_results(tlr_plan* p) {
  cudaStream_t s = p->stream;
  TRY(cuda_check(cudaMemcpyAsync(&p->hb->status, p->status, sizeof(int), cudaMemcpyDeviceToHost, s), "status"));
  TRY(cuda_check(cudaMemcpyAsync(p->hb->out, p->out, sizeof(double) * 3, cudaMemcpyDeviceToHost, s), "out"));
  TRY(cuda_check(cudaMemcpyAsync(p->hb->work, p->status + 4, sizeof(double) * 2 * TLR_NKINDS,
                                 cudaMemcpyDeviceToHost, s),
                 "work"));
  if (p->ntiles > 0) {
    TRY(cuda_check(cudaMemcpyAsync(p->h_rank, p->rank, sizeof(int) * p->ntiles, cudaMemcpyDeviceToHost, s),
                   "ranks"));
    TRY(cuda_check(cudaMemcpyAsync(p->h_rank0, p->rank0, sizeof(int) * p->ntiles, cudaMemcpyDeviceToHost, s),
                   "ranks0"));
  }
  return 0;
}

// Wait for the forward evaluation queued by enqueue_forward and report it (tlr_loglik's outputs).
int finish_forward(tlr_plan* p, double* loglik, tlr_info* info, int* factor_ranks, int* sigma_ranks) {
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  TRY(cuda_check(cudaStreamSynchronize(p->stream), "evaluation"));
  const int status = p->hb->status;
  if (p->prof) {
    for (size_t q = 0; q < p->ev_kind.size(); ++q) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p->ev_pool[2 * q], p->ev_pool[2 * q + 1]);
      p->kms[p->ev_kind[q]] += ms;
    }
  }
  p->ev_used = 0;
  p->ev_kind.clear();
  for (int q = 0; q < TLR_NKINDS; ++q) {
    p->kflops[q] += p->hb->work[2 * q];
    p->kbytes[q] += p->hb->work[2 * q + 1];
  }
  if (status < 0) {
    const char* why = status == TLR_ERR_RANK_CAP   ? "a tile rank exceeded the plan's rank capacity"
                      : status == TLR_ERR_COMPRESS ? "a tile needed more than 120 singular directions"
                      : status == TLR_ERR_TIMEOUT  ? "a device wait ran out of its iteration limit"
                                                   : "device error";
    return fail(status, why);
  }
  fill_info(p, status, p->hb->out, info, factor_ranks, sigma_ranks);
  if (loglik) *loglik = status == 0 ? p->hb->out[0] : NAN;
  p->factor_ok = status == 0;
  return status;
}

}  // namespace

extern "C" {

int tlr_loglik(tlr_plan* p, const double theta[3], int rule, double value, double* loglik, tlr_info* info,
               int* factor_ranks, int* sigma_ranks) {
  TRY(enqueue_forward(p, theta, rule, value));
  return finish_forward(p, loglik, info, factor_ranks, sigma_ranks);
}

int tlr_loglik_grad(tlr_plan* p, const double theta[3], int rule, double value, double* loglik, double* grad,
                    tlr_info* info, int* factor_ranks, int* sigma_ranks) {
  double ll = 0.0;
  const int rc = tlr_loglik(p, theta, rule, value, &ll, info, factor_ranks, sigma_ranks);
  if (loglik) *loglik = ll;
  if (rc != 0) return rc;
  double g[3] = {0.0, 0.0, 0.0};
  TRY(run_backward(p, theta[0], 1.0 / theta[1], theta[2]));
  TRY(finish_backward(p, g));
  if (grad)
    for (int a = 0; a < 3; ++a) grad[a] = g[a];
  return 0;
}

int tlr_loglik_grad_batch(tlr_plan* const* plans, int count, const double* thetas, int rule, double value,
                          double* loglik, double* grad, int* status) {
  if (!plans || !thetas || count < 0) return fail(TLR_ERR_ARG, "invalid arguments to tlr_loglik_grad_batch");
  for (int q = 0; q < count; ++q) {
    if (!plans[q]) return fail(TLR_ERR_ARG, "a plan of the batch is NULL");
    for (int r = 0; r < q; ++r)
      if (plans[r] == plans[q]) return fail(TLR_ERR_ARG, "a plan appears twice in the batch");
  }
  // every forward pass is queued before any is waited on: the plans' streams overlap on the GPU
  for (int q = 0; q < count; ++q) TRY(enqueue_forward(plans[q], thetas + 3 * q, rule, value));
  std::vector<int> st(count, 0);
  int first_error = 0;
  for (int q = 0; q < count; ++q) {
    double ll = NAN;
    const int rc = finish_forward(plans[q], &ll, nullptr, nullptr, nullptr);
    if (rc < 0 && !first_error) first_error = rc;
    st[q] = rc;
    if (loglik) loglik[q] = ll;
    // each backward pass is queued as soon as its forward pass is done, beside the later plans'
    // forward passes (after an error none is queued; those already queued finish on their streams)
    if (!first_error && rc == 0)
      TRY(run_backward(plans[q], thetas[3 * q], 1.0 / thetas[3 * q + 1], thetas[3 * q + 2]));
  }
  if (first_error) return first_error;
  for (int q = 0; q < count; ++q) {
    if (st[q] != 0) continue;
    double g[3];
    TRY(finish_backward(plans[q], g));
    if (grad)
      for (int a = 0; a < 3; ++a) grad[3 * q + a] = g[a];
  }
  if (status)
    for (int q = 0; q < count; ++q) status[q] = st[q];
  return 0;
}

int tlr_truncate_tiles(tlr_plan* p, const double theta[3], int rule, double value, double* K_dev, long long ldk,
                       tlr_tile_stats* stats, int* ranks) {
  if (!p || !theta) return fail(TLR_ERR_ARG, "invalid arguments to tlr_truncate_tiles");
  if (!p->has_data) return fail(TLR_ERR_NOT_READY, "tlr_set_data has not been called");
  if (rule != TLR_RULE_FIXED && rule != TLR_RULE_ADAPTIVE) return fail(TLR_ERR_ARG, "rule must be fixed or adaptive");
  if (p->pworld > 1) return fail(TLR_ERR_ARG, "the plan is partitioned");
  const double sigma2 = theta[0], range = theta[1], eta = theta[2];
  if (!(range > 0.0) || !std::isfinite(sigma2) || !std::isfinite(eta) || !std::isfinite(range))
    return fail(TLR_ERR_ARG, "theta must be finite with range > 0");
  p->round_store = 0;
  if (K_dev && ldk < p->n) return fail(TLR_ERR_ARG, "ldk must be at least N");
  if (K_dev && (long long)p->nB * (p->nB + 1) / 2 > 65535)
    return fail(TLR_ERR_ARG, "the dense write-out takes at most 361 tiles per side");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  cudaStream_t s = p->stream;
  p->factor_ok = false;
  LAUNCH(TLR_K_FILL, tlr::launch_set_params(p->status, make_params(p, theta, rule, value), s));
  TRY(cuda_check(cudaMemsetAsync(p->rank, 0, sizeof(int) * std::max(p->ntiles, 1), s), "reset ranks"));
  TRY(run_compression(p));
  if (K_dev)
    LAUNCH(TLR_K_GEN, tlr::launch_assemble(p->xy, p->n, p->b, sigma2, 1.0 / range, p->nu5, sigma2 * eta, p->U, p->V,
                                           p->rank, p->cap, K_dev, ldk, p->status, s));
  const size_t nt = (size_t)std::max(p->ntiles, 1);
  std::vector<double> tail(nt, 0.0), fro(nt, 0.0);
  TRY(cuda_check(cudaMemcpyAsync(&p->hb->status, p->status, sizeof(int), cudaMemcpyDeviceToHost, s), "status"));
  if (p->ntiles > 0) {
    TRY(cuda_check(cudaMemcpyAsync(p->h_rank0, p->rank, sizeof(int) * p->ntiles, cudaMemcpyDeviceToHost, s), "ranks"));
    TRY(cuda_check(cudaMemcpyAsync(tail.data(), p->tail0, sizeof(double) * p->ntiles, cudaMemcpyDeviceToHost, s),
                   "tails"));
    TRY(cuda_check(cudaMemcpyAsync(fro.data(), p->fro0, sizeof(double) * p->ntiles, cudaMemcpyDeviceToHost, s),
                   "norms"));
  }
  TRY(cuda_check(cudaStreamSynchronize(s), "truncate tiles"));
  const int status = p->hb->status;
  if (status < 0)
    return fail(status, status == TLR_ERR_RANK_CAP   ? "a tile rank exceeded the plan's rank capacity"
                        : status == TLR_ERR_COMPRESS ? "a tile needed more than 120 singular directions"
                                                     : "device error");
  // statistics as codes/11_tlr_rank_rules.py:83, 99-108
  const int nB = p->nB, b = p->b, n = p->n;
  auto bsz = [&](int i) { return std::min(b, n - i * b); };
  tlr_tile_stats st{};
  for (int i = 0; i < nB; ++i) st.stored += (long long)bsz(i) * bsz(i);
  double fro2 = 0.0;
  for (int i = 0; i < nB; ++i)
    for (int j = 0; j < i; ++j) {
      const int t = i * (i - 1) / 2 + j;
      const int r = p->h_rank0[t];
      st.stored += 2LL * r * std::max(bsz(i), bsz(j));
      st.max_rank = std::max(st.max_rank, r);
      fro2 += 2.0 * tail[t] * tail[t];
      st.max_abs = std::max(st.max_abs, tail[t]);
      st.max_rel = std::max(st.max_rel, tail[t] / std::max(fro[t], 1e-300));
      if (ranks) ranks[t] = r;
    }
  st.fro_err = std::sqrt(fro2);
  if (stats) *stats = st;
  return 0;
}

int tlr_loglik_host(tlr_plan* p, const double* xy_host, const double* y_host, const double theta[3], int rule,
                    double value, double* loglik, tlr_info* info, int* factor_ranks, int* sigma_ranks) {
  if (!p || !xy_host || !y_host) return fail(TLR_ERR_ARG, "invalid arguments to tlr_loglik_host");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  TRY(cuda_check(cudaMemcpyAsync(p->xy, xy_host, sizeof(double) * 2 * p->n, cudaMemcpyHostToDevice, p->stream),
                 "copy sites"));
  TRY(cuda_check(cudaMemcpyAsync(p->y, y_host, sizeof(double) * p->n, cudaMemcpyHostToDevice, p->stream),
                 "copy observations"));
  p->has_data = true;
  return tlr_loglik(p, theta, rule, value, loglik, info, factor_ranks, sigma_ranks);
}

int tlr_plan_set_precision(tlr_plan* p, int mode) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  if (mode != TLR_PRECISION_FP64 && mode != TLR_PRECISION_MIXED) return fail(TLR_ERR_ARG, "unknown precision mode");
  p->precision = mode;
  return 0;
}

int tlr_plan_rank_map(tlr_plan* p, int mode) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  if (mode != TLR_RANKS_RULE && mode != TLR_RANKS_RECORD && mode != TLR_RANKS_REPLAY)
    return fail(TLR_ERR_ARG, "rank map mode must be TLR_RANKS_RULE, TLR_RANKS_RECORD or TLR_RANKS_REPLAY");
  static_assert(TLR_RANKS_RECORD == tlr::kRankRecord && TLR_RANKS_REPLAY == tlr::kRankReplay, "rank map modes");
  p->rmode = mode;
  return 0;
}

long long tlr_plan_rank_map_size(const tlr_plan* p) { return p ? (long long)p->rlog_off[p->nB] : 0; }

int tlr_plan_rank_map_io(tlr_plan* p, int* ranks, int* bits, long long count, int upload) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  const size_t total = p->rlog_off[p->nB];
  if (count != (long long)total) return fail(TLR_ERR_ARG, "count must be tlr_plan_rank_map_size(plan)");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  TRY(cuda_check(cudaStreamSynchronize(p->stream), "rank map"));
  const auto kind = upload ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  if (ranks)
    TRY(cuda_check(upload ? cudaMemcpy(p->rlog, ranks, sizeof(int) * total, kind)
                          : cudaMemcpy(ranks, p->rlog, sizeof(int) * total, kind), "rank map ranks"));
  if (bits)  // the rounding decisions then the panel solves' (total + ntiles)
    TRY(cuda_check(upload ? cudaMemcpy(p->blog, bits, sizeof(int) * (total + p->ntiles), kind)
                          : cudaMemcpy(bits, p->blog, sizeof(int) * (total + p->ntiles), kind), "rank map bits"));
  return 0;
}

int tlr_factor_storage(tlr_plan* p, int* bits, long long* stored_bytes) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  if (!p->factor_ok) return fail(TLR_ERR_NOT_READY, "the plan holds no completed factorization");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  const int nB = p->nB, b = p->b, n = p->n;
  std::vector<int> pr((size_t)std::max(p->ntiles, 1), 64);
  if (p->round_store && p->ntiles > 0)
    TRY(cuda_check(cudaMemcpy(pr.data(), p->prec, sizeof(int) * p->ntiles, cudaMemcpyDeviceToHost), "bits"));
  auto bsz = [&](int i) { return std::min(b, n - i * b); };
  long long byt = 0;
  int q = 0;
  for (int k = 0; k < nB; ++k) byt += 8LL * bsz(k) * bsz(k);
  for (int k = 0; k < nB; ++k)
    for (int i = k + 1; i < nB; ++i) {
      const int t = i * (i - 1) / 2 + k;
      const int r = p->h_rank[t];
      const int bt = (p->round_store && r > 0) ? pr[t] : 64;
      byt += 2LL * r * bsz(i) * bt / 8;
      if (bits) bits[q++] = bt;
    }
  if (stored_bytes) *stored_bytes = byt;
  return 0;
}

int tlr_selftest_bounded_wait(long long iterations, int device, double* elapsed_ms, long long* limit) {
  if (limit) *limit = tlr::tc_wait_limit();
  if (iterations <= 0 || iterations > tlr::tc_wait_limit()) return fail(TLR_ERR_ARG, "iterations out of range");
  int rc = cuda_check(cudaSetDevice(device), "set device");
  if (rc) return rc;
  int* d = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int h = 1;
  rc = cuda_check(cudaMalloc(&d, sizeof(int)), "status word");
  if (!rc) rc = cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  if (!rc) rc = cuda_check(cudaEventCreate(&e0), "event");
  if (!rc) rc = cuda_check(cudaEventCreate(&e1), "event");
  if (!rc) rc = cuda_check(cudaEventRecord(e0, s), "event");
  if (!rc) rc = cuda_check((cudaError_t)tlr::launch_wait_selftest(iterations, d, s), "self-test launch");
  if (!rc) rc = cuda_check(cudaEventRecord(e1, s), "event");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s), "status copy");
  if (!rc) rc = cuda_check(cudaStreamSynchronize(s), "self-test");
  float ms = 0.f;
  if (!rc && elapsed_ms) {
    cudaEventElapsedTime(&ms, e0, e1);
    *elapsed_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (d) cudaFree(d);
  if (rc) return rc;
  if (h == TLR_ERR_TIMEOUT) return fail(TLR_ERR_TIMEOUT, "a device wait ran out of its iteration limit");
  return h;
}

int tlr_selftest_gemm(int precision, int transA, int transB, int M, int N, int K, double alpha, const double* A,
                      int lda, const double* B, int ldb, double beta, double* C, int ldc, int device) {
  if (precision != TLR_PRECISION_FP64 && precision != TLR_PRECISION_MIXED) return fail(TLR_ERR_ARG, "unknown precision");
  if (M < 0 || N < 0 || K < 0) return fail(TLR_ERR_ARG, "negative size");
  if (lda < std::max(1, transA ? K : M) || ldb < std::max(1, transB ? N : K) || ldc < std::max(1, M))
    return fail(TLR_ERR_ARG, "leading dimension too small");
  if ((M && N && !C) || (M && N && K && (!A || !B))) return fail(TLR_ERR_ARG, "NULL matrix");
  if (M == 0 || N == 0) return 0;
  int rc = cuda_check(cudaSetDevice(device), "set device");
  if (rc) return rc;
  const size_t status_bytes = sizeof(int) * (4 + 4 * TLR_NKINDS);
  tlr::GemmJob j{A, B, C, nullptr, lda, ldb, ldc, M, N, K, transA ? 1 : 0, transB ? 1 : 0, alpha, beta};
  TcSplitPlan sp;
  tc_split_plan(&j, 1, sp);
  // one buffer: job, operand pointers, split table, status, then the split area (16-byte aligned)
  const size_t oOps = 256, oSplit = 512, oStatus = 1024, oArea = 4096;
  unsigned char* d = nullptr;
  cudaStream_t s = nullptr;
  int h = 0;
  rc = cuda_check(cudaMalloc(&d, oArea + sizeof(float) * std::max<size_t>(sp.floats, 4)), "self-test buffers");
  if (rc) return rc;
  tlr::GemmJob* dj = reinterpret_cast<tlr::GemmJob*>(d);
  tlr::TcOperands* dops = reinterpret_cast<tlr::TcOperands*>(d + oOps);
  tlr::SplitJob* dsplit = reinterpret_cast<tlr::SplitJob*>(d + oSplit);
  int* st = reinterpret_cast<int*>(d + oStatus);
  float* area = reinterpret_cast<float*>(d + oArea);
  for (size_t q = 0; q < sp.splits.size(); ++q) sp.splits[q].dst = area + sp.split_off[q];
  tlr::TcOperands op{nullptr, nullptr};
  if (sp.job_off[0].first != SIZE_MAX) op = {area + sp.job_off[0].first, area + sp.job_off[0].second};
  rc = cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  if (!rc) rc = cuda_check(cudaMemsetAsync(st, 0, status_bytes, s), "status");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(dj, &j, sizeof(j), cudaMemcpyHostToDevice, s), "job");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(dops, &op, sizeof(op), cudaMemcpyHostToDevice, s), "operands");
  if (!rc && !sp.splits.empty())
    rc = cuda_check(cudaMemcpyAsync(dsplit, sp.splits.data(), sp.splits.size() * sizeof(tlr::SplitJob),
                                    cudaMemcpyHostToDevice, s),
                    "split table");
  if (!rc && precision == TLR_PRECISION_MIXED) {
    if (!sp.splits.empty())
      rc = cuda_check((cudaError_t)tlr::launch_split_tf32(dsplit, (int)sp.splits.size(), sp.max_blocks, st,
                                                          TLR_K_BWD_GEMM, s),
                      "split launch");
    if (!rc) rc = cuda_check((cudaError_t)tlr::launch_gemm_tc3(dj, dops, 1, M, N, st, TLR_K_BWD_GEMM, s), "gemm launch");
  } else if (!rc) {
    rc = cuda_check((cudaError_t)tlr::launch_dgemm_batched(dj, 1, M, N, st, TLR_K_BWD_GEMM, s), "gemm launch");
  }
  if (!rc) rc = cuda_check(cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, s), "status copy");
  if (!rc) rc = cuda_check(cudaStreamSynchronize(s), "self-test");
  if (s) cudaStreamDestroy(s);
  cudaFree(d);
  if (rc) return rc;
  if (h == TLR_ERR_TIMEOUT) return fail(TLR_ERR_TIMEOUT, "a device wait ran out of its iteration limit");
  return h;
}

int tlr_plan_set_kernel(tlr_plan* p, double nu) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  if (nu != 1.5 && nu != 2.5) return fail(TLR_ERR_ARG, "nu must be 1.5 or 2.5");
  p->nu5 = nu == 2.5 ? 1 : 0;
  return 0;
}

int tlr_plan_set_profiling(tlr_plan* p, int on) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  p->prof = on != 0;
  p->prof_kind = on < 0 ? -on - 1 : -1;  // on < 0: only the launches of kind -on - 1
  return 0;
}

int tlr_plan_set_graphs(tlr_plan* p, int on) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  p->use_graphs = on != 0;
  return 0;
}

// ------------------------------------------------------------------------------------------
// Block-row cyclic factorization (codes/13_multigpu_tile_cholesky.py:45-79 with the TLR tiles of
// codes/17_tlr_cholesky_pilot.py:137-215): the host runs the steps and moves the buffers.

int tlr_plan_set_partition(tlr_plan* p, int rank, int world) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  if (world < 1 || rank < 0 || rank >= world) return fail(TLR_ERR_ARG, "need 0 <= rank < world");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  TRY(cuda_check(cudaStreamSynchronize(p->stream), "partition"));
  if (world > 1 && !p->tmap) TRY(dalloc(p, &p->tmap, (size_t)std::max(p->ntiles, 1)));
  std::vector<int> own;
  for (int t = 0; t < p->ntiles; ++t)
    if (p->h_ti[t] % world == rank) own.push_back(t);
  if (world > 1 && !own.empty())
    TRY(cuda_check(cudaMemcpy(p->tmap, own.data(), sizeof(int) * own.size(), cudaMemcpyHostToDevice), "tile map"));
  p->prank = world > 1 ? rank : 0;
  p->pworld = world;
  p->nown = (int)own.size();
  p->factor_ok = false;
  return 0;
}

long long tlr_dist_buffer_doubles(const tlr_plan* p, int which, int k) {
  if (!p) return -1;
  if (which == TLR_DIST_DIAG) return 8 + (long long)p->b * p->b + p->b;
  if (which == TLR_DIST_PANEL) return (long long)tlr::dist_panel_doubles(p->b, p->cap, k, p->nB, p->pworld);
  if (which == TLR_DIST_SUMS) return 2LL * p->nB + p->ntiles + p->pworld;
  return -1;
}

namespace {
int dist_ready(tlr_plan* p, int k) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  if (k < 0 || k >= p->nB) return fail(TLR_ERR_ARG, "step out of range");
  return cuda_check(cudaSetDevice(p->device), "cudaSetDevice");
}

// Step k's diagonal tile on its owner: A_kk with the deferred updates, then POTRF and z_k.
int dist_diag(tlr_plan* p, int k, cudaStream_t st) {
  if (k % p->pworld != p->prank) return 0;
  LAUNCH_ON(st, TLR_K_DIAG, tlr::launch_diag_build(p->xy, p->n, p->b, k, p->U, p->Yd, p->rank, p->cap, p->D,
                                                   p->status, st));
  LAUNCH_ON(st, TLR_K_POTRF, tlr::launch_potrf(p->D, p->n, p->b, k, p->rhs, p->z, p->ldpart, p->qpart, p->status,
                                               st));
  return 0;
}
}  // namespace

int tlr_dist_begin(tlr_plan* p, const double theta[3], int rule, double value) {
  if (!p || !theta) return fail(TLR_ERR_ARG, "invalid arguments to tlr_dist_begin");
  if (!p->has_data) return fail(TLR_ERR_NOT_READY, "tlr_set_data has not been called");
  if (rule != TLR_RULE_FIXED && rule != TLR_RULE_ADAPTIVE)
    return fail(TLR_ERR_ARG, "the partitioned factorization takes the fixed and adaptive rules");
  if (p->rmode != tlr::kRankOff) return fail(TLR_ERR_ARG, "the partitioned factorization keeps no rank map");
  const double sigma2 = theta[0], range = theta[1], eta = theta[2];
  if (!(range > 0.0) || !std::isfinite(sigma2) || !std::isfinite(eta) || !std::isfinite(range))
    return fail(TLR_ERR_ARG, "theta must be finite with range > 0");
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  cudaStream_t s = p->stream;
  p->factor_ok = false;
  p->round_store = 0;
  LAUNCH(TLR_K_FILL, tlr::launch_set_params(p->status, make_params(p, theta, rule, value), s));
  TRY(cuda_check(cudaMemsetAsync(p->rank, 0, sizeof(int) * std::max(p->ntiles, 1), s), "reset ranks"));
  TRY(cuda_check(cudaMemsetAsync(p->ldpart, 0, sizeof(double) * p->nB, s), "log det parts"));
  TRY(cuda_check(cudaMemsetAsync(p->qpart, 0, sizeof(double) * p->nB, s), "quadratic parts"));
  TRY(cuda_check(cudaMemsetAsync(p->rc_next, 0, sizeof(int) * p->nB, s), "pair counters"));
  TRY(cuda_check(cudaMemcpyAsync(p->rhs, p->y, sizeof(double) * p->n, cudaMemcpyDeviceToDevice, s), "rhs"));
  TRY(run_compression(p));
  if (p->ntiles > 0)
    TRY(cuda_check(cudaMemcpyAsync(p->rank0, p->rank, sizeof(int) * p->ntiles, cudaMemcpyDeviceToDevice, s),
                   "rank0"));
  return dist_diag(p, 0, s);
}

int tlr_dist_pack_diag(tlr_plan* p, int k, double* buf) {
  TRY(dist_ready(p, k));
  if (!buf) return fail(TLR_ERR_ARG, "buffer is NULL");
  LAUNCH(TLR_K_FILL, tlr::launch_dist_pack_diag(p->D, p->z, p->status, p->n, p->b, k, buf, p->stream));
  return 0;
}

int tlr_dist_unpack_diag(tlr_plan* p, int k, const double* buf) {
  TRY(dist_ready(p, k));
  if (!buf) return fail(TLR_ERR_ARG, "buffer is NULL");
  if (k % p->pworld == p->prank) return 0;  // the owner keeps its own
  LAUNCH(TLR_K_FILL, tlr::launch_dist_unpack_diag(p->D, p->z, p->status, p->n, p->b, k, buf, p->stream));
  return 0;
}

int tlr_dist_solve_step(tlr_plan* p, int k) {
  TRY(dist_ready(p, k));
  LAUNCH(TLR_K_TRSM, tlr::launch_trsm(p->D, p->n, p->b, k, p->nB, p->U, p->V, p->Wd, p->Yd, p->rank, p->cap, p->z,
                                      p->rhs, p->prec, p->blog + p->rlog_off[p->nB], p->prank, p->pworld, p->status,
                                      p->stream));
  return 0;
}

int tlr_dist_pack_panel(tlr_plan* p, int k, double* buf) {
  TRY(dist_ready(p, k));
  if (!buf) return fail(TLR_ERR_ARG, "buffer is NULL");
  LAUNCH(TLR_K_FILL, tlr::launch_dist_pack_panel(p->U, p->V, p->rank, p->status, p->n, p->b, k, p->nB, p->cap,
                                                 p->prank, p->pworld, buf, p->stream));
  return 0;
}

int tlr_dist_unpack_panel(tlr_plan* p, int k, const double* gathered) {
  TRY(dist_ready(p, k));
  if (!gathered) return fail(TLR_ERR_ARG, "buffer is NULL");
  if (p->pworld == 1) return 0;
  const size_t len = tlr::dist_panel_doubles(p->b, p->cap, k, p->nB, p->pworld);
  LAUNCH(TLR_K_FILL, tlr::launch_dist_unpack_panel(p->U, p->V, p->rank, p->status, p->n, p->b, k, p->nB, p->cap,
                                                   p->prank, p->pworld, gathered, len, p->stream));
  return 0;
}

int tlr_dist_update_step(tlr_plan* p, int k) {
  TRY(dist_ready(p, k));
  cudaStream_t s = p->stream, sd = p->side;
  const bool ahead = k + 1 < p->nB && (k + 1) % p->pworld == p->prank;
  if (ahead) {  // the next diagonal tile on the side stream, beside this step's recompression
    TRY(cuda_check(cudaEventRecord(p->ev_panel, s), "event"));
    TRY(cuda_check(cudaStreamWaitEvent(sd, p->ev_panel, 0), "wait"));
    TRY(dist_diag(p, k + 1, sd));
    TRY(cuda_check(cudaEventRecord(p->ev_diag, sd), "event"));
  }
  LAUNCH(TLR_K_RECOMPRESS, tlr::launch_recompress(p->n, p->b, k, p->nB, p->U, p->V, p->rank, p->cap, p->rcs,
                                                  p->slot_doubles, p->nslots, p->rc_next + k, p->rlog + p->rlog_off[k],
                                                  p->blog + p->rlog_off[k], p->prank, p->pworld, p->status, s));
  if (ahead) TRY(cuda_check(cudaStreamWaitEvent(s, p->ev_diag, 0), "wait"));
  return 0;
}

int tlr_dist_pack_sums(tlr_plan* p, double* buf) {
  TRY(dist_ready(p, 0));
  if (!buf) return fail(TLR_ERR_ARG, "buffer is NULL");
  LAUNCH(TLR_K_FILL, tlr::launch_dist_pack_sums(p->ldpart, p->qpart, p->rank0, p->ti, p->status, p->nB, p->ntiles,
                                                p->prank, p->pworld, buf, p->stream));
  return 0;
}

int tlr_dist_finish(tlr_plan* p, const double* sums, double* loglik, tlr_info* info, int* factor_ranks,
                    int* sigma_ranks) {
  TRY(dist_ready(p, 0));
  if (!sums) return fail(TLR_ERR_ARG, "buffer is NULL");
  cudaStream_t s = p->stream;
  LAUNCH(TLR_K_FILL, tlr::launch_dist_unpack_sums(p->ldpart, p->qpart, p->rank0, p->status, p->nB, p->ntiles,
                                                  p->pworld, sums, s));
  LAUNCH(TLR_K_FINISH, tlr::launch_finish(p->nB, p->n, p->ldpart, p->qpart, p->out, p->status, s));
  TRY(enqueue_results(p));
  const int rc = finish_forward(p, loglik, info, factor_ranks, sigma_ranks);
  p->factor_ok = false;  // each rank holds its own block rows only
  return rc;
}

int tlr_plan_kernel_stats(tlr_plan* p, double* ms, long long* launches, double* flops, double* bytes, int nkinds,
                          int reset) {
  if (!p) return fail(TLR_ERR_ARG, "plan is NULL");
  for (int q = 0; q < nkinds && q < TLR_NKINDS; ++q) {
    if (ms) ms[q] = p->kms[q];
    if (launches) launches[q] = p->klaunch[q];
    if (flops) flops[q] = p->kflops[q];
    if (bytes) bytes[q] = p->kbytes[q];
  }
  if (reset)
    for (int q = 0; q < TLR_NKINDS; ++q) {
      p->kms[q] = 0.0;
      p->klaunch[q] = 0;
      p->kflops[q] = 0.0;
      p->kbytes[q] = 0.0;
    }
  return 0;
}

int tlr_factor_solve(tlr_plan* p, double* x_dev, int m, int trans) {
  if (!p || !x_dev || m < 0 || (trans != 0 && trans != 1)) return fail(TLR_ERR_ARG, "invalid arguments to tlr_factor_solve");
  if (!p->factor_ok) return fail(TLR_ERR_NOT_READY, "the plan holds no completed factorization");
  if (m == 0) return 0;
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  const int rc = tlr::launch_factor_solve(p->D, p->U, p->V, p->rank, p->cap, p->n, p->b, p->nB, x_dev, m, trans,
                                          p->stream);
  if (rc) return fail(TLR_ERR_CUDA, std::string("solve launch: ") + cudaGetErrorString((cudaError_t)rc));
  return cuda_check(cudaStreamSynchronize(p->stream), "solve");
}

int tlr_factor_matvec(tlr_plan* p, const double* z_dev, double* y_dev, int m) {
  if (!p || !z_dev || !y_dev || m < 0 || z_dev == y_dev)
    return fail(TLR_ERR_ARG, "invalid arguments to tlr_factor_matvec");
  if (!p->factor_ok) return fail(TLR_ERR_NOT_READY, "the plan holds no completed factorization");
  if (m == 0) return 0;
  TRY(cuda_check(cudaSetDevice(p->device), "cudaSetDevice"));
  const int rc = tlr::launch_factor_matvec(p->D, p->U, p->V, p->rank, p->cap, p->n, p->b, p->nB, z_dev, y_dev, m,
                                           p->stream);
  if (rc) return fail(TLR_ERR_CUDA, std::string("matvec launch: ") + cudaGetErrorString((cudaError_t)rc));
  return cuda_check(cudaStreamSynchronize(p->stream), "matvec");
}

int tlr_get_diag_tile(tlr_plan* p, int k, double* out_host) {
  if (!p || !out_host || k < 0 || k >= p->nB) return fail(TLR_ERR_ARG, "invalid arguments to tlr_get_diag_tile");
  const int bk = std::min(p->b, p->n - k * p->b);
  std::vector<double> tmp((size_t)p->b * p->b);
  TRY(cuda_check(cudaMemcpyAsync(tmp.data(), p->D + (size_t)k * p->b * p->b, sizeof(double) * p->b * p->b,
                                 cudaMemcpyDeviceToHost, p->stream),
                 "copy diag"));
  TRY(cuda_check(cudaStreamSynchronize(p->stream), "sync"));
  for (int c = 0; c < bk; ++c)
    for (int a = 0; a < bk; ++a) out_host[(size_t)c * bk + a] = a >= c ? tmp[(size_t)c * p->b + a] : 0.0;
  return 0;
}

int tlr_get_offdiag_tile(tlr_plan* p, int i, int j, double* u_host, double* v_host, int* rank) {
  if (!p || i <= j || j < 0 || i >= p->nB) return fail(TLR_ERR_ARG, "invalid tile index");
  const int t = i * (i - 1) / 2 + j;
  int r = 0;
  TRY(cuda_check(cudaMemcpyAsync(&r, p->rank + t, sizeof(int), cudaMemcpyDeviceToHost, p->stream), "rank"));
  TRY(cuda_check(cudaStreamSynchronize(p->stream), "sync"));
  if (rank) *rank = r;
  const int bi = std::min(p->b, p->n - i * p->b), bj = std::min(p->b, p->n - j * p->b);
  std::vector<double> tu((size_t)p->b * p->cap), tv((size_t)p->b * p->cap);
  TRY(cuda_check(cudaMemcpyAsync(tu.data(), p->U + (size_t)t * p->b * p->cap, sizeof(double) * p->b * p->cap,
                                 cudaMemcpyDeviceToHost, p->stream), "copy U"));
  TRY(cuda_check(cudaMemcpyAsync(tv.data(), p->V + (size_t)t * p->b * p->cap, sizeof(double) * p->b * p->cap,
                                 cudaMemcpyDeviceToHost, p->stream), "copy V"));
  TRY(cuda_check(cudaStreamSynchronize(p->stream), "sync"));
  for (int c = 0; c < r; ++c) {
    if (u_host)
      for (int a = 0; a < bi; ++a) u_host[(size_t)c * bi + a] = tu[(size_t)c * p->b + a];
    if (v_host)
      for (int a = 0; a < bj; ++a) v_host[(size_t)c * bj + a] = tv[(size_t)c * p->b + a];
  }
  return 0;
}

}  // extern "C"
