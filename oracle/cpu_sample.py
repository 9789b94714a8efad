"""Sampled CPU timing of the reference TLR pipeline (TEST / BASELINE INFRASTRUCTURE ONLY).

One evaluation of the reference's tlr_loglik (codes/17_tlr_cholesky_pilot.py:259) at N = 50,000,
b = 500 takes about five minutes on an 8-core host, too long for a benchmark step.  This module
times the reference's own per-tile operations, as restated in oracle/tlr_oracle.py (NumPy/SciPy,
the same LAPACK calls), on a bounded random sample of the real tiles of the evaluation and
scales each by the number of times one evaluation performs it:

  truncate_svd of an off-diagonal tile (with its generation)   x  nB (nB - 1) / 2
  cholesky of a diagonal tile (with its generation)            x  nB
  solve_triangular of a panel tile                             x  nB (nB - 1) / 2
  diagonal rank-r update                                       x  nB (nB - 1) / 2
  recompress of a trailing tile (with W, U_ik W, hstack)       x  sum_k (nB-k-1)(nB-k-2)/2
  tile forward-solve update                                    x  nB (nB - 1) / 2

The recompression samples are step-0 updates of randomly chosen pairs (i, j); their ranks are the
initial ranks, close to the factor ranks seen later in the factorization.  The result is an
estimate of seconds per evaluation, stated as such.
"""
from __future__ import annotations

import time

import numpy as np
from scipy.linalg import cholesky, solve_triangular

from . import tlr_oracle as O


class SampledPipeline:
    def __init__(self, S, y, theta, b, rule, value, n_pairs=64, seed=0):
        self.S, self.y = S, y
        self.theta = tuple(float(v) for v in theta)
        self.n = S.shape[0]
        self.b = b
        self.bounds = O.tile_bounds(self.n, b)
        self.nB = len(self.bounds)
        self.rule, self.value = rule, value
        self.thr_rel, self.thr_abs = O.thresholds(self.n, max(e - s for s, e in self.bounds), self.theta, rule, value)
        rng = np.random.default_rng(seed)
        nB = self.nB
        # setup (untimed): diagonal tile 0, its Cholesky, the compressed panel column 0, and the
        # trailing tiles of a random set of step-0 pairs
        self.L00 = cholesky(self._diag(0), lower=True, check_finite=False)
        self.panel = {i: self._compress(i, 0)[:2] for i in range(1, nB)}
        self.panel_solved = {}
        for i, (U, V) in self.panel.items():
            if U.shape[1]:
                V = solve_triangular(self.L00, V, lower=True, check_finite=False)
            self.panel_solved[i] = (U, V)
        pairs = [(i, j) for i in range(2, nB) for j in range(1, i)]
        pick = rng.choice(len(pairs), size=min(n_pairs, len(pairs)), replace=False)
        self.pairs = [pairs[q] for q in pick]
        self.trailing = {p: self._compress(*p)[:2] for p in self.pairs}
        self.counts = dict(compress=nB * (nB - 1) // 2, potrf=nB, trsm=nB * (nB - 1) // 2,
                           diag=nB * (nB - 1) // 2, solve=nB * (nB - 1) // 2,
                           recompress=sum((nB - k - 1) * (nB - k - 2) // 2 for k in range(nB)))

    def _block(self, i, j):
        (i0, i1), (j0, j1) = self.bounds[i], self.bounds[j]
        sigma2, rg, _ = self.theta
        return sigma2 * O.matern32(O.pairwise_dist(self.S[i0:i1], self.S[j0:j1]), rg)

    def _diag(self, k):
        D = self._block(k, k)
        D[np.diag_indices_from(D)] += self.theta[0] * self.theta[2]
        return D

    def _compress(self, i, j):
        U, V, tail, r = O.truncate_svd(self._block(i, j), self.rule, self.thr_rel, self.thr_abs)
        return U, V, r

    def step(self, n_compress=8, n_trsm=16, n_recompress=32, seed=1):
        """Time one bounded sample; return (estimated seconds per evaluation, sample seconds)."""
        rng = np.random.default_rng(seed)
        nB = self.nB
        t_all = time.perf_counter()
        # initial compression
        tiles = [(int(i), int(rng.integers(0, i))) for i in rng.integers(1, nB, size=n_compress)]
        t0 = time.perf_counter()
        for i, j in tiles:
            self._compress(i, j)
        t_comp = (time.perf_counter() - t0) / n_compress
        # diagonal generation + POTRF
        t0 = time.perf_counter()
        cholesky(self._diag(int(rng.integers(0, nB))), lower=True, check_finite=False)
        t_potrf = time.perf_counter() - t0
        # panel TRSM, diagonal update and forward-solve update
        idx = [int(q) for q in rng.integers(1, nB, size=n_trsm)]
        z0 = solve_triangular(self.L00, self.y[: self.bounds[0][1]], lower=True, check_finite=False)
        t_trsm = t_diag = t_solve = 0.0
        for i in idx:
            U, V = self.panel[i]
            t0 = time.perf_counter()
            if U.shape[1]:
                V = solve_triangular(self.L00, V, lower=True, check_finite=False)
            t1 = time.perf_counter()
            if U.shape[1]:
                D = np.empty((U.shape[0], U.shape[0]))
                W = V.T @ V
                D -= (U @ W) @ U.T
            t2 = time.perf_counter()
            if U.shape[1]:
                _ = U @ (V.T @ z0)
            t3 = time.perf_counter()
            t_trsm += t1 - t0
            t_diag += t2 - t1
            t_solve += t3 - t2
        t_trsm /= n_trsm
        t_diag /= n_trsm
        t_solve /= n_trsm
        # Schur update + recompression of step-0 pairs
        sel = [self.pairs[int(q)] for q in rng.integers(0, len(self.pairs), size=n_recompress)]
        t0 = time.perf_counter()
        for i, j in sel:
            Ui, Vi = self.panel_solved[i]
            Uj, Vj = self.panel_solved[j]
            if Ui.shape[1] == 0 or Uj.shape[1] == 0:
                continue
            W = Vi.T @ Vj
            Uij, Vij = self.trailing[(i, j)]
            O.recompress(np.hstack([Uij, -(Ui @ W)]), np.hstack([Vij, Uj]), self.rule, self.thr_rel, self.thr_abs)
        t_rc = (time.perf_counter() - t0) / n_recompress
        c = self.counts
        est = (c["compress"] * t_comp + c["potrf"] * t_potrf + c["trsm"] * t_trsm + c["diag"] * t_diag
               + c["solve"] * t_solve + c["recompress"] * t_rc)
        return est, time.perf_counter() - t_all


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        n = [p.get("num_threads", 1) for p in threadpool_info() if p.get("user_api") == "blas"]
        return int(max(n)) if n else 1
    except Exception:
        return 1


def timed_full_evaluation(S, y, theta, b, rule, value, steps):
    """One complete evaluation of the reference pipeline (oracle.tlr_loglik: tile generation and
    compression, the right-looking TLR Cholesky, the forward solve; codes/17_tlr_cholesky_pilot.py:
    137-266), timed stage by stage.  The 2 nB + 1 stages (nB compression rows, nB factorization
    steps, the solve) are dealt into `steps` consecutive groups of nearly equal count; a group's
    time is the sum of its stages' times, so the groups add up to the measured evaluation.

    Returns dict(seconds, step_seconds, loglik, completed, stages)."""
    bounds = O.tile_bounds(S.shape[0], b)
    marks = []
    t0 = time.perf_counter()
    ll, _, info = O.tlr_loglik(S, y, tuple(float(v) for v in theta), bounds, rule, value,
                               on_stage=lambda lab: marks.append(time.perf_counter()))
    t1 = time.perf_counter()
    marks.append(t1)  # the solve (or the end of a failed factorization)
    stage_s = np.diff(np.concatenate(([t0], marks)))
    nst = len(stage_s)
    steps = max(1, min(int(steps), nst))
    group = (np.arange(nst) * steps) // nst
    step_s = [float(stage_s[group == q].sum()) for q in range(steps)]
    return dict(seconds=t1 - t0, step_seconds=step_s, loglik=ll, completed=bool(info.get("completed", False)),
                stages=nst)
