"""Reference-facing Python surface of the B200 TLR log-likelihood.

Mirrors the functions the pilot scripts call (marysalvana/adaptive-tlr-pilots):

  tile_bounds(n, b)                         codes/11_tlr_rank_rules.py:69-71
  morton_order(xy, order=10)                codes/11_tlr_rank_rules.py:40-53   (on the GPU)
  tlr_loglik(S, y, theta, bounds, rule, v)  codes/17_tlr_cholesky_pilot.py:259-266
  neg_loglik_tlr(logth, S, y, bounds, ...)  codes/17_tlr_cholesky_pilot.py:279-290
  make_cov, neg_loglik (assembled rule)     codes/11_tlr_rank_rules.py:74-138
  Likelihood(S, y, b, device, svd_mode)     codes/19_tlr_mcmc_gpu.py:27-138 (assembled Sigma^TLR)
  loglik(theta, locs, y, b, rule, tau|eps)  the (loglik, per-tile ranks, PD) form

Every evaluation runs on the GPU through libtlr_b200.so (include/tlr_b200.h).  There is no CPU
path: without the library or a CUDA device these functions raise.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import _lib

RULES = {"fixed": _lib.TLR_RULE_FIXED, "adaptive": _lib.TLR_RULE_ADAPTIVE, "mixed": _lib.TLR_RULE_MIXED}
STORAGE_BITS = (8, 16, 32, 64)
KERNELS = (1.5, 2.5)  # Matern smoothness nu
_NU = 1.5


def set_kernel(nu):
    """Covariance smoothness for every later evaluation of plans that have none of their own:
    nu = 1.5 (Matern 3/2, the default) or 2.5 (Matern 5/2).  The counterpart of
    codes/24_screening_stress.py:46-47 set_kernel, which patches the kernel of 17 globally."""
    global _NU
    if float(nu) not in KERNELS:
        raise ValueError(f"nu must be one of {KERNELS}")
    _NU = float(nu)


def get_kernel():
    return _NU


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("adaptive_tlr_pilots_b200 needs a CUDA device (no CPU fallback)")
    return torch


def tile_bounds(n, b):
    """[(0, b), (b, 2b), ..., (., n)]; the last tile may be short (codes/11_tlr_rank_rules.py:69-71)."""
    edges = list(range(0, n, b)) + [n]
    return [(edges[t], edges[t + 1]) for t in range(len(edges) - 1)]


def _tile_size(bounds, n):
    """The uniform tile size of a bounds list made by tile_bounds; ValueError otherwise."""
    if not bounds:
        raise ValueError("bounds is empty")
    b = bounds[0][1] - bounds[0][0]
    if b <= 0 or list(map(tuple, bounds)) != tile_bounds(n, b):
        raise ValueError("bounds must be tile_bounds(n, b) for one tile size b")
    return b


def morton_order(xy, order=10, device=0):
    """Stable Z-order permutation of points (N x 2), computed on the GPU.

    Same quantisation, bit interleave and stable tie order as codes/11_tlr_rank_rules.py:40-53."""
    torch = _torch()
    xy = np.ascontiguousarray(np.asarray(xy, dtype=np.float64))
    if xy.ndim != 2 or xy.shape[1] != 2:
        raise ValueError("xy must be N x 2")
    n = xy.shape[0]
    lib = _lib.load()
    dev = torch.device("cuda", device)
    with torch.cuda.device(dev):
        t = torch.from_numpy(xy).to(dev)
        perm = torch.empty(n, dtype=torch.int64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.tlr_morton_order(ctypes.c_void_p(t.data_ptr()), n, order, ctypes.c_void_p(perm.data_ptr()),
                                        ctypes.c_void_p(stream)))
        return perm.cpu().numpy()


@dataclass
class Evaluation:
    status: int                 # 0 ok, k + 1 not PD at diagonal tile k
    loglik: float | None
    info: dict
    factor_ranks: np.ndarray    # reference L_off order (for k, for i > k)
    sigma_ranks: np.ndarray     # initial ranks (for i, for j < i)
    grad: np.ndarray | None = None  # d loglik / d(sigma2, range, eta), when requested


class Plan:
    """Device workspace for one (N, b) problem: owns a tlr_plan of the C ABI."""

    MAX_CAP = 128  # the C plan's largest rank capacity

    def __init__(self, n, b, cap=64, device=0):
        torch = _torch()
        self.lib = _lib.load()
        self.n, self.b, self.cap, self.device = int(n), int(b), int(cap), int(device)
        self.nB = (self.n + self.b - 1) // self.b
        self.ntiles = self.nB * (self.nB - 1) // 2
        self.dev = torch.device("cuda", self.device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.handle = None
        self.generation = 0
        self._data = None
        self.precision = "fp64"
        self.graphs = True      # forward pass replayed from a CUDA graph (set_graphs)
        self.nu = None          # None: follow set_kernel; else this plan's own smoothness
        self._create()

    def _create(self):
        h = ctypes.c_void_p()
        _lib.check(self.lib.tlr_plan_create(ctypes.byref(h), self.n, self.b, self.cap, self.device,
                                            ctypes.c_void_p(self.stream.cuda_stream)))
        self.handle = h
        self._nu_applied = 1.5  # the C plan starts with Matern 3/2

    def grow(self, cap=None):
        """Recreate the device workspace with a larger rank capacity (default: double, at most
        MAX_CAP), keeping the loaded data, precision and kernel.  Returns False when the capacity
        is already the largest."""
        new = min(self.MAX_CAP, int(cap) if cap is not None else 2 * self.cap)
        if new <= self.cap:
            return False
        self.close()
        self.cap = new
        self._create()
        if self.precision != "fp64":
            _lib.check(self.lib.tlr_plan_set_precision(self.handle, _lib.PRECISIONS[self.precision]))
        if not getattr(self, "graphs", True):
            _lib.check(self.lib.tlr_plan_set_graphs(self.handle, 0))
        if getattr(self, "partition", (0, 1))[1] > 1:
            self.set_partition(*self.partition)
        self._apply_kernel()
        if getattr(self, "rank_mode", "rule") != "rule":
            # a recorded map does not survive the new workspace: record again
            self.rank_map("record")
        if self._data is not None:
            S_t, y_t = self._data
            _lib.check(self.lib.tlr_set_data(self.handle, ctypes.c_void_p(S_t.data_ptr()),
                                             ctypes.c_void_p(y_t.data_ptr())))
        self.generation += 1
        return True

    def set_kernel(self, nu):
        """This plan's covariance smoothness (1.5 or 2.5), independent of set_kernel."""
        if float(nu) not in KERNELS:
            raise ValueError(f"nu must be one of {KERNELS}")
        self.nu = float(nu)
        self._apply_kernel()

    def _apply_kernel(self):
        nu = self.nu if self.nu is not None else _NU
        if nu != self._nu_applied:
            _lib.check(self.lib.tlr_plan_set_kernel(self.handle, ctypes.c_double(nu)))
            self._nu_applied = nu

    def close(self):
        if self.handle is not None and self.handle.value:
            self.lib.tlr_plan_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_data(self, S, y):
        """Load Morton-ordered sites and observations (numpy or torch) onto the device.  The copies
        run on the plan's stream after the work queued so far on the current stream (which may
        have produced device inputs)."""
        torch = _torch()
        self.stream.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(self.stream):
            S_t = torch.as_tensor(S, dtype=torch.float64).to(self.dev).contiguous()
            y_t = torch.as_tensor(y, dtype=torch.float64).to(self.dev).contiguous()
        if S_t.shape != (self.n, 2) or y_t.shape != (self.n,):
            raise ValueError(f"expected S of shape ({self.n}, 2) and y of shape ({self.n},)")
        self._data = (S_t, y_t)
        _lib.check(self.lib.tlr_set_data(self.handle, ctypes.c_void_p(S_t.data_ptr()),
                                         ctypes.c_void_p(y_t.data_ptr())))

    def evaluate(self, theta, rule, value, host_S=None, host_y=None, grad=False) -> Evaluation:
        """One log-likelihood evaluation (and its gradient when grad=True) on the device.

        A tile rank above the plan's capacity does not end the call: the workspace is recreated
        with twice the capacity (up to MAX_CAP) and the evaluation repeated, so the call succeeds
        wherever the reference's does, up to ranks of MAX_CAP."""
        while True:
            try:
                return self._evaluate(theta, rule, value, host_S, host_y, grad)
            except _lib.TlrError as e:
                if e.code != _lib.ERR_RANK_CAP or not self.grow():
                    raise

    def _evaluate(self, theta, rule, value, host_S, host_y, grad) -> Evaluation:
        if rule not in RULES:
            raise ValueError(f"rule must be one of {sorted(RULES)}, got {rule!r}")
        self._apply_kernel()
        th = (ctypes.c_double * 3)(*[float(v) for v in theta])
        ll = ctypes.c_double(0.0)
        info = _lib.TlrInfo()
        fr = np.zeros(max(self.ntiles, 1), dtype=np.int32)
        sr = np.zeros(max(self.ntiles, 1), dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        g = (ctypes.c_double * 3)()
        if grad:
            if host_S is not None:
                self.set_data(host_S, host_y)
            rc = self.lib.tlr_loglik_grad(self.handle, th, RULES[rule], float(value), ctypes.byref(ll), g,
                                          ctypes.byref(info), fr.ctypes.data_as(ip), sr.ctypes.data_as(ip))
        elif host_S is not None:
            S = np.ascontiguousarray(host_S, dtype=np.float64)
            y = np.ascontiguousarray(host_y, dtype=np.float64)
            if S.shape != (self.n, 2) or y.shape != (self.n,):
                raise ValueError(f"expected S of shape ({self.n}, 2) and y of shape ({self.n},)")
            rc = self.lib.tlr_loglik_host(self.handle, S.ctypes.data_as(ctypes.c_void_p),
                                          y.ctypes.data_as(ctypes.c_void_p), th, RULES[rule], float(value),
                                          ctypes.byref(ll), ctypes.byref(info), fr.ctypes.data_as(ip),
                                          sr.ctypes.data_as(ip))
        else:
            rc = self.lib.tlr_loglik(self.handle, th, RULES[rule], float(value), ctypes.byref(ll), ctypes.byref(info),
                                     fr.ctypes.data_as(ip), sr.ctypes.data_as(ip))
        rc = _lib.check(rc)
        self.generation += 1
        d = dict(completed=bool(info.completed), stored_sigma=int(info.stored_sigma),
                 max_rank_sigma=int(info.max_rank_sigma))
        if rc == 0:
            d.update(stored_factor=int(info.stored_factor), mean_rank_factor=float(info.mean_rank_factor),
                     max_rank_factor=int(info.max_rank_factor), logdet=float(info.logdet), quad=float(info.quad))
            if rule == "mixed":  # the storage bookkeeping of codes/17_tlr_cholesky_pilot.py:210-214
                bits = np.zeros(max(self.ntiles, 1), dtype=np.int32)
                byt = ctypes.c_longlong(0)
                _lib.check(self.lib.tlr_factor_storage(self.handle, bits.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                       ctypes.byref(byt)))
                bits = [int(v) for v in bits[: self.ntiles]]
                dense = self.n * (self.n + 1) // 2 * 8
                d.update(stored_factor_bytes=int(byt.value), dense_factor_bytes=dense,
                         factor_bytes_frac=byt.value / dense, factor_prec=bits,
                         precision_mix_factor_tiles={q: bits.count(q) for q in STORAGE_BITS})
        else:
            d.update(failed_at=int(info.failed_at))
        return Evaluation(rc, float(ll.value) if rc == 0 else None, d, fr[: self.ntiles], sr[: self.ntiles],
                          np.array(list(g)) if (grad and rc == 0) else None)

    def set_precision(self, mode="fp64"):
        """'fp64' (the parity path) or 'mixed' (tensor-core 3xTF32 backward GEMMs)."""
        if mode not in _lib.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_lib.PRECISIONS)}")
        _lib.check(self.lib.tlr_plan_set_precision(self.handle, _lib.PRECISIONS[mode]))
        self.precision = mode

    def truncate_tiles(self, theta, rule, value, assemble=False):
        """The assembled-matrix rule on the loaded sites (codes/11_tlr_rank_rules.py:74-108):
        (stats, ranks, K) with stats = dict(stored, max_rel, max_abs, fro_err, max_rank), the
        initial ranks in the order (i, j < i), and K the dense Sigma^TLR as a device tensor
        (assemble=True) or None.  Leaves no factor in the plan.  A rank above the capacity grows
        the plan, as evaluate does."""
        torch = _torch()
        if rule not in RULES:
            raise ValueError(f"rule must be one of {sorted(RULES)}, got {rule!r}")
        while True:
            self._apply_kernel()
            K = torch.empty((self.n, self.n), dtype=torch.float64, device=self.dev) if assemble else None
            th = (ctypes.c_double * 3)(*[float(v) for v in theta])
            st = _lib.TlrTileStats()
            rk = np.zeros(max(self.ntiles, 1), dtype=np.int32)
            try:
                _lib.check(self.lib.tlr_truncate_tiles(self.handle, th, RULES[rule], float(value),
                                                       ctypes.c_void_p(K.data_ptr() if K is not None else 0),
                                                       self.n, ctypes.byref(st),
                                                       rk.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
                break
            except _lib.TlrError as e:
                del K
                if e.code != _lib.ERR_RANK_CAP or not self.grow():
                    raise
        self.generation += 1
        stats = dict(stored=int(st.stored), max_rel=float(st.max_rel), max_abs=float(st.max_abs),
                     fro_err=float(st.fro_err), max_rank=int(st.max_rank))
        return stats, rk[: self.ntiles], K

    def rank_map(self, mode):
        """'rule' (the rule picks every rank), 'record' (and they are recorded) or 'replay' (the
        recorded ranks replace the rule's: frozen ranks at another theta)."""
        if mode not in _lib.RANK_MAP:
            raise ValueError(f"rank map mode must be one of {sorted(_lib.RANK_MAP)}")
        _lib.check(self.lib.tlr_plan_rank_map(self.handle, _lib.RANK_MAP[mode]))
        self.rank_mode = mode

    def rank_map_get(self):
        """(ranks, bits) of the plan's rank map (tlr_plan_rank_map_io): every recorded rank, and
        under rule 'mixed' the storage bits of every rounding, then those of the panel solves."""
        m = int(self.lib.tlr_plan_rank_map_size(self.handle))
        ranks = np.zeros(max(m, 1), dtype=np.int32)
        bits = np.zeros(max(m + self.ntiles, 1), dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.check(self.lib.tlr_plan_rank_map_io(self.handle, ranks.ctypes.data_as(ip), bits.ctypes.data_as(ip), m, 0))
        return ranks[:m], bits[: m + self.ntiles]

    def rank_map_set(self, ranks, bits=None):
        """Load a rank map (and storage bits) for later rank_map('replay') evaluations."""
        m = int(self.lib.tlr_plan_rank_map_size(self.handle))
        r = np.ascontiguousarray(ranks, dtype=np.int32)
        if r.shape != (m,):
            raise ValueError(f"ranks must hold {m} values")
        ip = ctypes.POINTER(ctypes.c_int)
        bp = None
        if bits is not None:
            bb = np.ascontiguousarray(bits, dtype=np.int32)
            if bb.shape != (m + self.ntiles,):
                raise ValueError(f"bits must hold {m + self.ntiles} values")
            bp = bb.ctypes.data_as(ip)
        _lib.check(self.lib.tlr_plan_rank_map_io(self.handle, r.ctypes.data_as(ip), bp, m, 1))

    def set_profiling(self, on=True, kind=None):
        """Bracket every launch with CUDA events (per-kernel device time; results unchanged), or
        only the launches of one kernel kind (a key of kernel_stats) when `kind` is given."""
        code = (-(_lib.KERNEL_KINDS.index(kind) + 1) if kind is not None else 1) if on else 0
        _lib.check(self.lib.tlr_plan_set_profiling(self.handle, code))

    def set_partition(self, rank, world):
        """Hold block rows i with i % world == rank only (the block-row cyclic factorization of
        blockrow.py; world = 1 lifts it).  A partitioned plan is evaluated through blockrow."""
        _lib.check(self.lib.tlr_plan_set_partition(self.handle, int(rank), int(world)))
        self.partition = (int(rank), int(world))

    def set_graphs(self, on=True):
        """Replay the forward pass from a CUDA graph captured once per precision (default), or
        issue its launches one by one (off).  Results are bit-identical either way."""
        _lib.check(self.lib.tlr_plan_set_graphs(self.handle, 1 if on else 0))
        self.graphs = bool(on)

    def kernel_stats(self, reset=False):
        """{kernel kind: dict(ms, launches, flops, bytes)} accumulated since the last reset
        (ms needs profiling on; flops/bytes are the kernels' own algorithmic counts)."""
        nk = len(_lib.KERNEL_KINDS)
        ms = (ctypes.c_double * nk)()
        cnt = (ctypes.c_longlong * nk)()
        fl = (ctypes.c_double * nk)()
        by = (ctypes.c_double * nk)()
        _lib.check(self.lib.tlr_plan_kernel_stats(self.handle, ms, cnt, fl, by, nk, 1 if reset else 0))
        return {k: dict(ms=ms[q], launches=cnt[q], flops=fl[q], bytes=by[q]) for q, k in enumerate(_lib.KERNEL_KINDS)}

    # products and solves with the factor of the last successful evaluation (device, in place)
    def _cols(self, X):
        torch = _torch()
        X = torch.as_tensor(X, dtype=torch.float64, device=self.dev)
        squeeze = X.dim() == 1
        X2 = X[:, None] if squeeze else X
        if X2.shape[0] != self.n:
            raise ValueError(f"expected {self.n} rows")
        return X2.t().contiguous().clone(), squeeze  # column-major n x m storage = row-major m x n

    def solve(self, B, trans=False):
        """L^{-1} B (trans False) or L^{-T} B (trans True) on the device; B n or n x m."""
        Xt, squeeze = self._cols(B)
        _lib.check(self.lib.tlr_factor_solve(self.handle, ctypes.c_void_p(Xt.data_ptr()), Xt.shape[0],
                                             1 if trans else 0))
        X = Xt.t()
        return X[:, 0] if squeeze else X

    def matvec_L(self, Z):
        """L Z on the device; Z n or n x m."""
        Zt, squeeze = self._cols(Z)
        Yt = _torch().empty_like(Zt)
        _lib.check(self.lib.tlr_factor_matvec(self.handle, ctypes.c_void_p(Zt.data_ptr()),
                                              ctypes.c_void_p(Yt.data_ptr()), Zt.shape[0]))
        Y = Yt.t()
        return Y[:, 0] if squeeze else Y

    # factor access (checking / prediction)
    def diag_tile(self, k):
        bk = min(self.b, self.n - k * self.b)
        out = np.zeros((bk, bk), order="F")
        _lib.check(self.lib.tlr_get_diag_tile(self.handle, k, out.ctypes.data_as(ctypes.c_void_p)))
        return np.ascontiguousarray(out)

    def offdiag_tile(self, i, j):
        bi = min(self.b, self.n - i * self.b)
        bj = min(self.b, self.n - j * self.b)
        u = np.zeros((self.cap, bi))
        v = np.zeros((self.cap, bj))
        r = ctypes.c_int(0)
        _lib.check(self.lib.tlr_get_offdiag_tile(self.handle, i, j, u.ctypes.data_as(ctypes.c_void_p),
                                                 v.ctypes.data_as(ctypes.c_void_p), ctypes.byref(r)))
        r = r.value
        return np.ascontiguousarray(u[:r].T), np.ascontiguousarray(v[:r].T)


class PlanBatch:
    """Batched evaluation of `count` parameter vectors on one device, sharing the sites and
    observations: evaluate(thetas) runs batched calls (tlr_loglik_grad_batch) in which every
    workspace's forward pass is queued before any is waited on, so the GPU overlaps the plans'
    latency-bound factorization steps.  The batch of MCMC chains or optimizer restarts of one
    iteration.

    `workspaces` (default: count, at most count; "auto": the autotuner's measured best) is the
    number of device workspaces (plans, one stream each) that run at once; with fewer workspaces than parameter vectors the vectors go
    through them in consecutive groups, so memory is workspaces x (one plan) whatever the count
    (at N = 50,000, b = 500 a plan holds about 10 GB: 64 chains through 8 workspaces fit one
    B200)."""

    def __init__(self, n, b, count, cap=64, device=0, precision="mixed", workspaces=None):
        torch = _torch()
        self.n, self.b, self.count, self.device = int(n), int(b), int(count), int(device)
        if workspaces == "auto":  # the autotuner's table (adaptive_tlr_pilots_b200/autotune.py)
            from .autotune import best_workspaces
            workspaces = best_workspaces(self.n, self.b, self.count, precision=precision)
        self.workspaces = self.count if workspaces is None else max(1, min(int(workspaces), self.count))
        self.lib = _lib.load()
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(self.workspaces)]
        self.plans = []
        for st in self.streams:
            with torch.cuda.stream(st):
                p = Plan(self.n, self.b, cap, self.device)
            p.set_precision(precision)
            self.plans.append(p)
        self.nB = self.plans[0].nB

    def set_data(self, S, y):
        """One host-to-device copy (numpy or torch, pinned host memory welcome), then a device copy
        into every plan."""
        torch = _torch()
        dev = torch.device("cuda", self.device)
        S_t = torch.as_tensor(S, dtype=torch.float64).to(dev, non_blocking=True).contiguous()
        y_t = torch.as_tensor(y, dtype=torch.float64).to(dev, non_blocking=True).contiguous()
        if S_t.shape != (self.n, 2) or y_t.shape != (self.n,):
            raise ValueError(f"expected S of shape ({self.n}, 2) and y of shape ({self.n},)")
        torch.cuda.current_stream(dev).synchronize()
        for p in self.plans:
            p._data = (S_t, y_t)
            _lib.check(p.lib.tlr_set_data(p.handle, ctypes.c_void_p(S_t.data_ptr()), ctypes.c_void_p(y_t.data_ptr())))

    def evaluate(self, thetas, rule, value):
        """[(loglik | None, grad | None, status)] for up to `count` parameter vectors, in groups of
        `workspaces`.  A rank above the plans' capacity grows every plan (Plan.grow) and repeats
        the group."""
        th = np.atleast_2d(np.asarray(thetas, dtype=np.float64))
        if th.shape[0] > self.count or th.shape[1] != 3:
            raise ValueError(f"thetas must be at most {self.count} x 3")
        out = []
        for g0 in range(0, th.shape[0], self.workspaces):
            grp = th[g0:g0 + self.workspaces]
            while True:
                try:
                    out.extend(self._evaluate(grp, rule, value))
                    break
                except _lib.TlrError as e:
                    if e.code != _lib.ERR_RANK_CAP or not all([p.grow() for p in self.plans]):
                        raise
        return out

    def _evaluate(self, thetas, rule, value):
        if rule not in RULES:
            raise ValueError(f"rule must be one of {sorted(RULES)}, got {rule!r}")
        th = np.ascontiguousarray(np.atleast_2d(np.asarray(thetas, dtype=np.float64)))
        m = th.shape[0]
        if m > self.workspaces or th.shape[1] != 3:
            raise ValueError(f"at most {self.workspaces} parameter vectors per batched call")
        for p in self.plans[:m]:
            p._apply_kernel()
        handles = (ctypes.c_void_p * m)(*[p.handle.value for p in self.plans[:m]])
        ll = np.full(m, np.nan)
        g = np.zeros((m, 3))
        st = np.zeros(m, dtype=np.int32)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(self.lib.tlr_loglik_grad_batch(handles, m, th.ctypes.data_as(dp), RULES[rule], float(value),
                                                  ll.ctypes.data_as(dp), g.ctypes.data_as(dp),
                                                  st.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        for p in self.plans[:m]:
            p.generation += 1
        return [(float(ll[q]) if st[q] == 0 else None, g[q].copy() if st[q] == 0 else None, int(st[q]))
                for q in range(m)]

    def close(self):
        for p in self.plans:
            p.close()
        self.plans = []


class TLRFactor:
    """Lazy view of the factor left in a plan by the last evaluation (L_diag, L_off as in
    codes/17_tlr_cholesky_pilot.py:215).  Invalidated by the plan's next evaluation."""

    def __init__(self, plan: Plan):
        self.plan = plan
        self.generation = plan.generation

    def _check(self):
        if self.plan.generation != self.generation:
            raise RuntimeError("this factor was overwritten by a later evaluation on the same plan")

    @property
    def L_diag(self):
        self._check()
        return [self.plan.diag_tile(k) for k in range(self.plan.nB)]

    def forward(self, B):
        """Solve L X = B on the device (codes/17_tlr_cholesky_pilot.py:230-240 tlr_forward)."""
        self._check()
        return self.plan.solve(B, trans=False)

    def backward(self, Z):
        """Solve L^T X = Z on the device (17:243-256 tlr_backward)."""
        self._check()
        return self.plan.solve(Z, trans=True)

    def matvec(self, Z):
        """L Z on the device (17:218-227 tlr_matvec_L)."""
        self._check()
        return self.plan.matvec_L(Z)

    @property
    def L_off(self):
        self._check()
        out = {}
        for k in range(self.plan.nB):
            for i in range(k + 1, self.plan.nB):
                out[(i, k)] = self.plan.offdiag_tile(i, k)
        return out


_PLANS: dict = {}


def get_plan(n, b, cap=64, device=0) -> Plan:
    key = (int(n), int(b), int(cap), int(device))
    p = _PLANS.get(key)
    if p is None:
        p = Plan(n, b, cap, device)
        _PLANS[key] = p
    return p


def release_plans():
    for p in _PLANS.values():
        p.close()
    _PLANS.clear()


class TLRLogLik:
    """torch.autograd.Function over the plan: loglik(theta) with d loglik / d theta from the
    hand-written backward kernels (ranks frozen at theta).  The backward kernels run inside the
    forward call, while the factor is on the device; backward() only scales the stored gradient."""

    _fn = None

    @classmethod
    def function(cls):
        if cls._fn is None:
            import torch

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, theta, plan, rule, value):
                    ev = plan.evaluate(theta.detach().cpu().tolist(), rule, value, grad=True)
                    if ev.status != 0:
                        out = torch.tensor(float("-inf"), dtype=torch.float64)
                        ctx.save_for_backward(torch.zeros(3, dtype=torch.float64))
                        return out
                    ctx.save_for_backward(torch.tensor(ev.grad, dtype=torch.float64))
                    return torch.tensor(ev.loglik, dtype=torch.float64)

                @staticmethod
                def backward(ctx, g):
                    (grad,) = ctx.saved_tensors
                    return g * grad, None, None, None

            cls._fn = _Fn
        return cls._fn

    @classmethod
    def apply(cls, theta, plan, rule, value):
        return cls.function().apply(theta, plan, rule, value)


def tlr_loglik_grad(S, y, theta, bounds, rule, value, cap=64, device=0, precision="fp64"):
    """(loglik | None, gradient | None, info): the log-likelihood of tlr_loglik and its gradient
    in (sigma2, range, eta) from the device backward pass.  precision 'fp64' (every step in FP64)
    or 'mixed' (tensor-core products where the accuracy budget allows)."""
    S = np.asarray(S, dtype=np.float64)
    n = S.shape[0]
    b = _tile_size(bounds, n)
    plan = get_plan(n, b, cap, device)
    plan.set_precision(precision)
    ev = plan.evaluate(theta, rule, value, host_S=S, host_y=np.asarray(y, dtype=np.float64), grad=True)
    if ev.status != 0:
        return None, None, ev.info
    return ev.loglik, ev.grad, ev.info


def tlr_loglik(S, y, theta, bounds, rule, value, cap=64, device=0, precision="fp64"):
    """Drop-in for codes/17_tlr_cholesky_pilot.py:259 tlr_loglik.

    Returns (loglik, factor, info) or (None, None, info) when a diagonal tile is not positive
    definite (info['completed'] False, info['failed_at'] = k), like 17:172-176.  `factor` is a
    lazy TLRFactor on the device.  precision 'fp64' is the reference's arithmetic (the default);
    'mixed' is the mixed-precision path."""
    S = np.asarray(S, dtype=np.float64)
    n = S.shape[0]
    b = _tile_size(bounds, n)
    plan = get_plan(n, b, cap, device)
    plan.set_precision(precision)
    ev = plan.evaluate(theta, rule, value, host_S=S, host_y=np.asarray(y, dtype=np.float64))
    if ev.status != 0:
        return None, None, ev.info
    return ev.loglik, TLRFactor(plan), ev.info


def _cross_cov(Sp, S, theta, device=0, nu=1.5):
    """sigma2 * matern(dist(Sp, S)) on the device (np x n), codes/17_tlr_cholesky_pilot.py:270
    (nu = 2.5: the kernel of codes/24_screening_stress.py:38-42)."""
    torch = _torch()
    dev = torch.device("cuda", device)
    A = torch.as_tensor(np.asarray(Sp, dtype=np.float64), device=dev)
    B = torch.as_tensor(np.asarray(S, dtype=np.float64), device=dev)
    if nu == 2.5:
        x = torch.cdist(A, B) * ((5.0 ** 0.5) / float(theta[1]))
        return float(theta[0]) * (1.0 + x + x * x / 3.0) * torch.exp(-x)
    x = torch.cdist(A, B) * ((3.0 ** 0.5) / float(theta[1]))
    return float(theta[0]) * (1.0 + x) * torch.exp(-x)


def tlr_predict(S, y, Sp, theta, bounds, fac):
    """Kriging mean and standard deviation at Sp with the TLR factor (drop-in for
    codes/17_tlr_cholesky_pilot.py:269-276): alpha = L^-T L^-1 y, mu = Kp alpha, W = L^-1 Kp^T,
    var = sigma2 (1 + eta) - colsum(W^2).  The solves run on the device through the C ABI."""
    torch = _torch()
    fac._check()
    plan = fac.plan
    Kp = _cross_cov(Sp, S, theta, plan.device, plan._nu_applied)
    yt = torch.as_tensor(np.asarray(y, dtype=np.float64), device=plan.dev)
    alpha = fac.backward(fac.forward(yt))
    mu = Kp @ alpha
    W = fac.forward(Kp.t())
    var = float(theta[0]) * (1.0 + float(theta[2])) - (W * W).sum(0)
    return mu.cpu().numpy(), torch.sqrt(torch.clamp(var, min=1e-12)).cpu().numpy()


def skill(yp, mu, sig):
    """RMSE, CRPS of the Gaussian predictive and 90% coverage (codes/11_tlr_rank_rules.py:142-165)."""
    from math import erf, pi, sqrt
    yp, mu, sig = (np.asarray(v, dtype=np.float64) for v in (yp, mu, sig))
    z = (yp - mu) / sig
    pdf = np.exp(-0.5 * z ** 2) / sqrt(2 * pi)
    cdf = 0.5 * (1 + np.vectorize(erf)(z / sqrt(2)))
    crps = float((sig * (z * (2 * cdf - 1) + 2 * pdf - 1 / sqrt(pi))).mean())
    return dict(rmse=float(np.sqrt(((yp - mu) ** 2).mean())), crps=crps, cover90=float((np.abs(z) <= 1.6448536).mean()))


def neg_loglik_tlr(logth, S, y, bounds, rule, value, trace):
    """Optimizer objective, codes/17_tlr_cholesky_pilot.py:279-290: 1e12 on a failed
    factorization, evaluations and failures counted in `trace`."""
    theta = np.exp(logth)
    trace["evals"] += 1
    if rule == "dense":
        ll = dense_loglik(S, y, theta)
    else:
        ll, _, _ = tlr_loglik(S, y, theta, bounds, rule, value)
    if ll is None:
        trace["failures"] += 1
        return 1e12
    return -ll


def dense_loglik(S, y, theta, device=0):
    """Dense FP64 log-likelihood on the GPU (cuSOLVER Cholesky through torch); None if not PD.

    The 'dense' rule of codes/17_tlr_cholesky_pilot.py:282-284 (rules.loglik_dense, 11:112-120),
    with the kernel chosen by set_kernel."""
    torch = _torch()
    dev = torch.device("cuda", device)
    St = torch.as_tensor(np.asarray(S, dtype=np.float64), device=dev)
    yt = torch.as_tensor(np.asarray(y, dtype=np.float64), device=dev)
    sigma2, rng, eta = [float(v) for v in theta]
    with torch.no_grad():
        K = torch.cdist(St, St)
        if _NU == 2.5:  # (1 + x + x^2 / 3) e^{-x}, x = sqrt(5) h / range
            K.mul_((5.0 ** 0.5) / rng)
            E = torch.exp(-K)
            K.mul_(K.div(3.0).add_(1.0)).add_(1.0).mul_(E).mul_(sigma2)
        else:
            K.mul_((3.0 ** 0.5) / rng)
            E = torch.exp(-K)
            K.add_(1.0).mul_(E).mul_(sigma2)
        del E
        K.diagonal().add_(sigma2 * eta)
        L, info = torch.linalg.cholesky_ex(K)
        del K
        if int(info.item()) != 0:
            return None
        z = torch.linalg.solve_triangular(L, yt[:, None], upper=False)[:, 0]
        ld = 2.0 * torch.log(torch.diagonal(L)).sum()
        out = float(-0.5 * (z @ z + ld + len(yt) * np.log(2 * np.pi)))
        del L
    return out


def loglik(theta, locs, y, b, rule, tau=None, eps=None, ordered=False, cap=64, device=0):
    """(loglik | None, per-tile factor ranks, PD flag) for sites `locs` and observations `y`.

    rule 'adaptive' takes tau, rule 'fixed' takes eps.  Unless ordered=True the sites are first
    put into Morton order on the GPU (the reference orders them before every fit, 17:324)."""
    if rule == "adaptive":
        if tau is None:
            raise ValueError("rule 'adaptive' needs tau")
        value = tau
    elif rule == "fixed":
        if eps is None:
            raise ValueError("rule 'fixed' needs eps")
        value = eps
    else:
        raise ValueError(f"rule must be 'adaptive' or 'fixed', got {rule!r}")
    locs = np.asarray(locs, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if not ordered:
        perm = morton_order(locs, device=device)
        locs, y = locs[perm], y[perm]
    n = locs.shape[0]
    plan = get_plan(n, b, cap, device)
    plan.set_precision("fp64")
    ev = plan.evaluate(theta, rule, value, host_S=locs, host_y=y)
    return ev.loglik, ev.factor_ranks.copy(), ev.status == 0


def _dense_cov(S, theta, device=0):
    """Dense Sigma(theta) = sigma2 M + sigma2 eta I on the device (codes/11_tlr_rank_rules.py:61-65),
    with the kernel chosen by set_kernel."""
    torch = _torch()
    dev = torch.device("cuda", device)
    St = torch.as_tensor(np.asarray(S, dtype=np.float64), device=dev)
    sigma2, rng, eta = [float(v) for v in theta]
    with torch.no_grad():
        K = torch.cdist(St, St)
        if _NU == 2.5:
            K.mul_((5.0 ** 0.5) / rng)
            E = torch.exp(-K)
            K.mul_(K.div(3.0).add_(1.0)).add_(1.0).mul_(E).mul_(sigma2)
        else:
            K.mul_((3.0 ** 0.5) / rng)
            E = torch.exp(-K)
            K.add_(1.0).mul_(E).mul_(sigma2)
        del E
        K.diagonal().add_(sigma2 * eta)
    return K


def make_cov(S, theta, rule, value, bounds, device=0, cap=64):
    """(K, info): Sigma(theta) on the device, with every off-diagonal tile truncated under the rule
    for rule 'fixed' / 'adaptive' (info = (stored, max_rel, max_abs, ||Sigma - Sigma^TLR||_F,
    ranks), the return of truncate_tiles), or exact for rule 'dense' (info None).  Drop-in for
    codes/11_tlr_rank_rules.py:121-126 make_cov with truncate_tiles (11:74-108) inside; S must be
    Morton-ordered and bounds = tile_bounds(N, b)."""
    S = np.asarray(S, dtype=np.float64)
    if rule == "dense":
        return _dense_cov(S, theta, device), None
    n = S.shape[0]
    b = _tile_size(bounds, n)
    plan = get_plan(n, b, cap, device)
    plan.set_data(S, np.zeros(n))
    st, ranks, K = plan.truncate_tiles(theta, rule, value, assemble=True)
    return K, (st["stored"], st["max_rel"], st["max_abs"], st["fro_err"], [int(r) for r in ranks])


def loglik_dense_K(K, y):
    """(loglik, L) of y under the dense device matrix K, or (None, None) when K is not positive
    definite: codes/11_tlr_rank_rules.py:112-120 loglik_dense, the Cholesky on the device."""
    torch = _torch()
    with torch.no_grad():
        yt = torch.as_tensor(np.asarray(y, dtype=np.float64), device=K.device)
        L, info = torch.linalg.cholesky_ex(K)
        if int(info.item()) != 0:
            return None, None
        z = torch.linalg.solve_triangular(L, yt[:, None], upper=False)[:, 0]
        ld = 2.0 * torch.log(torch.diagonal(L)).sum()
        return float(-0.5 * (z @ z + ld + len(yt) * np.log(2 * np.pi))), L


def neg_loglik(logth, S, y, rule, value, bounds, trace, device=0):
    """Negative log-likelihood of the assembled-matrix rule at exp(logth), 1e12 when Sigma^TLR is
    not positive definite: codes/11_tlr_rank_rules.py:130-138 (trace counts evals and failures)."""
    theta = np.exp(np.asarray(logth, dtype=np.float64))
    K, _ = make_cov(S, theta, rule, value, bounds, device=device)
    ll, _ = loglik_dense_K(K, y)
    del K
    trace["evals"] += 1
    if ll is None:
        trace["failures"] += 1
        return 1e12
    return -ll


class Likelihood:
    """codes/19_tlr_mcmc_gpu.py:27-138: Likelihood(S, y, b, device, svd_mode=...)(theta, rule, value)
    is the log-likelihood of y under Sigma^TLR(theta), the covariance with every off-diagonal tile
    truncated under the rule (assembled densely on the device), through a dense Cholesky; -inf
    when that Cholesky fails; self.last = dict(ok, stored, time, L).  rule 'dense' skips the
    truncation.

    svd_mode: the reference offers 'fp64' (exact batched SVD, the minimal rank meeting the rule),
    'fp32' and 'rand' (ranks whose FP64-verified error meets the rule, possibly above the minimal
    one).  Here every mode uses the device compression (randomized sketch, exact FP64 residual,
    widened until the rank is resolved), which gives the minimal ranks of 'fp64'; so the ranks are
    those of 'fp64' in all three modes and never above the reference's 'fp32' / 'rand' ones.
    rand_k, rand_power and seed are accepted for the call surface; last_fallback is always 0."""

    MODES = ("fp64", "fp32", "rand")

    def __init__(self, S, y, b, device=0, dtype=None, svd_mode="fp32", rand_k=64, rand_power=2, seed=0, cap=64):
        if svd_mode not in self.MODES:
            raise ValueError(f"svd_mode must be one of {self.MODES}")
        self.svd_mode, self.rand_k, self.rand_power, self.last_fallback = svd_mode, rand_k, rand_power, 0
        self.n = int(np.asarray(S).shape[0])
        self.b = int(b)
        dev = device.index if hasattr(device, "index") and device.index is not None else (
            0 if not isinstance(device, int) else device)
        self.device = dev
        self.S = np.asarray(S, dtype=np.float64)
        self.y = np.asarray(y, dtype=np.float64)
        self.plan = Plan(self.n, self.b, cap, dev)
        self.plan.set_data(self.S, self.y)
        self.last = {}

    def __call__(self, theta, rule, value):
        torch = _torch()
        t0 = time.time()
        if rule == "dense":
            K, stored = _dense_cov(self.S, theta, self.device), self.n * self.n
        else:
            st, _, K = self.plan.truncate_tiles(theta, rule, value, assemble=True)
            stored = st["stored"]
        ll, L = loglik_dense_K(K, self.y)
        del K
        torch.cuda.synchronize(self.device)
        ok = ll is not None
        self.last = dict(ok=ok, stored=stored, time=time.time() - t0, L=L)
        return ll if ok else -float("inf")
