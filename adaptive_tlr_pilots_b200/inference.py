"""Inference drivers on the B200 TLR likelihood: maximum likelihood with the device gradient,
observed information, multi-chain MCMC (random-walk Metropolis and gradient-based MALA) with
checkpoint/resume, and the reference's multi-chain diagnostics.

Reference counterparts (marysalvana/adaptive-tlr-pilots):
  mle                   codes/17_tlr_cholesky_pilot.py:377-401 (Nelder-Mead on log theta from
                        theta_true * (1.5, 0.6, 2.0); here L-BFGS-B with the analytic gradient)
  observed_information  codes/15_pilot_standard_errors.py:21-31, 55-57 (central differences of the
                        log-likelihood; here central differences of the device gradient)
  run_chains            codes/19_tlr_mcmc_gpu.py:170-202 and codes/38_tlr_cholesky_mcmc.py:89-135
                        (random-walk Metropolis on log theta in the prior box, Robbins-Monro scale
                        adaptation to acceptance 0.3, checkpoints every 100 iterations); the
                        chains advance in lockstep so that one iteration is one batch of
                        likelihood evaluations
  split_rhat_ess        codes/35_mcmc_multichain_diagnostics.py:26-59 (rank-normalised split R-hat
                        and bulk ESS of Vehtari et al. 2021)
The objective takes any callable evaluator, so the samplers and the optimizer are testable on the
CPU with an analytic density; on the GPU the evaluator is a TLR plan (:class:`TLRObjective`).
"""
from __future__ import annotations

import os
import time

import numpy as np

# prior box on log(sigma2, range, eta): codes/19_tlr_mcmc_gpu.py:23
LO = np.log([0.1, 0.02, 0.001])
HI = np.log([10.0, 2.0, 1.0])


class TLRObjective:
    """Log-likelihood (and gradient) in x = log(theta) on one GPU plan.

    __call__(x, grad) -> (ll, g) with g = d ll / d x = theta * d ll / d theta; ll = -inf and g =
    None when the factorization fails (a diagonal tile is not positive definite).
    batch(X, grad) evaluates many parameter vectors: with batch=B > 1 through B plans and the
    batched entry point (tlr_loglik_grad_batch), B vectors per call; `workspaces` < B runs them
    through that many device workspaces in groups (PlanBatch), bounding the memory."""

    def __init__(self, S, y, b, rule, value, precision="mixed", cap=64, device=0, batch=1, workspaces=None):
        from .tlr import Plan, PlanBatch
        S = np.asarray(S, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        self.plan = Plan(S.shape[0], b, cap, device)
        self.plan.set_data(S, y)
        self.plan.set_precision(precision)
        self.pbatch = None
        if batch > 1:
            self.pbatch = PlanBatch(S.shape[0], b, batch, cap, device, precision, workspaces=workspaces)
            self.pbatch.set_data(S, y)
        self.rule, self.value = rule, value
        self.evals = 0

    def __call__(self, x, grad=True):
        theta = np.exp(np.asarray(x, dtype=np.float64))
        ev = self.plan.evaluate(theta, self.rule, self.value, grad=grad)
        self.evals += 1
        if ev.status != 0:
            return -np.inf, None
        return ev.loglik, (ev.grad * theta if grad else None)

    def batch(self, X, grad=True):
        X = np.atleast_2d(np.asarray(X, dtype=np.float64))
        ll = np.full(len(X), -np.inf)
        g = np.zeros((len(X), 3))
        if self.pbatch is not None:  # one batched call per `batch` parameter vectors
            B = self.pbatch.count
            for q0 in range(0, len(X), B):
                for q, (l, gr, st) in enumerate(self.pbatch.evaluate(np.exp(X[q0:q0 + B]), self.rule, self.value)):
                    if st == 0:
                        ll[q0 + q] = l
                        g[q0 + q] = gr * np.exp(X[q0 + q])
        else:
            for q, x in enumerate(X):
                e = self.plan.evaluate(np.exp(x), self.rule, self.value, grad=grad)
                if e.status == 0:
                    ll[q] = e.loglik
                    if grad:
                        g[q] = e.grad * np.exp(x)
        self.evals += len(X)
        return ll, (g if grad else None)

    def close(self):
        self.plan.close()
        if self.pbatch is not None:
            self.pbatch.close()


def _batch(obj, X, grad):
    if hasattr(obj, "batch"):
        return obj.batch(X, grad)
    out = [obj(x, grad) for x in X]
    ll = np.array([o[0] for o in out])
    g = np.array([o[1] if o[1] is not None else np.zeros(len(x)) for o, x in zip(out, X)]) if grad else None
    return ll, g


# ------------------------------------------------------------------------------------------ MLE
def mle(obj, x0, maxiter=200, gtol=1e-5, box=(LO, HI)):
    """Maximum likelihood in x = log(theta) by L-BFGS-B with the analytic gradient.

    A failed factorization returns the reference's penalty 1e12 (codes/17_tlr_cholesky_pilot.py:
    288-289) with a zero gradient; failures are counted.  When one stops the line search, the
    search continues from the best point with Nelder-Mead (the reference's optimizer) and is
    polished by L-BFGS-B again."""
    from scipy import optimize
    trace = dict(evals=0, failures=0, best_f=np.inf, best_x=np.asarray(x0, dtype=np.float64))

    def f(x):
        trace["evals"] += 1
        ll, g = obj(x, True)
        if not np.isfinite(ll):
            trace["failures"] += 1
            return 1e12, np.zeros_like(x)
        if -ll < trace["best_f"]:
            trace["best_f"], trace["best_x"] = -ll, np.array(x)
        return -ll, -np.asarray(g)

    t0 = time.time()
    bnds = list(zip(box[0], box[1]))
    res = optimize.minimize(f, np.asarray(x0, dtype=np.float64), jac=True, method="L-BFGS-B", bounds=bnds,
                            options=dict(maxiter=maxiter, gtol=gtol))
    if not res.success and trace["failures"]:
        # a failed factorization stopped the line search: continue from the best point with the
        # reference's derivative-free method on the same penalised objective, then polish
        res = optimize.minimize(lambda x: f(x)[0], trace["best_x"], method="Nelder-Mead", bounds=bnds,
                                options=dict(xatol=1e-7, fatol=1e-9, maxiter=40 * maxiter))
        res = optimize.minimize(f, res.x, jac=True, method="L-BFGS-B", bounds=bnds,
                                options=dict(maxiter=maxiter, gtol=gtol))
        if not res.success and trace["best_f"] <= res.fun:
            res.x = trace["best_x"]
    ll, g = obj(res.x, True)
    return dict(theta_hat=np.exp(res.x).tolist(), x_hat=res.x.tolist(), loglik=float(ll),
                grad_log=None if g is None else np.asarray(g).tolist(), evals=trace["evals"],
                failures=trace["failures"], success=bool(res.success), message=str(res.message),
                seconds=time.time() - t0)


def observed_information(obj, x, h=1e-4):
    """Observed information (negative Hessian of the log-likelihood) in x = log(theta) by central
    differences of the analytic gradient, symmetrised; with standard errors on both scales
    (SE_theta = theta * SE_log, as codes/15_pilot_standard_errors.py:55-57)."""
    x = np.asarray(x, dtype=np.float64)
    p = len(x)
    H = np.zeros((p, p))
    X = []
    for i in range(p):
        e = np.zeros(p)
        e[i] = h
        X += [x + e, x - e]
    ll, G = _batch(obj, np.array(X), True)
    if not np.all(np.isfinite(ll)):
        raise RuntimeError("a factorization failed inside the finite-difference stencil")
    for i in range(p):
        H[:, i] = (G[2 * i] - G[2 * i + 1]) / (2 * h)
    H = 0.5 * (H + H.T)
    info = -H
    cov = np.linalg.inv(info)
    se_log = np.sqrt(np.maximum(np.diag(cov), 0.0))
    return dict(info_log=info, cov_log=cov, se_log=se_log, se_theta=np.exp(x) * se_log)


# ----------------------------------------------------------------------------------------- MCMC
class ChainState:
    """State of M chains advancing in lockstep (log-theta scale)."""

    def __init__(self, starts, iters, seeds, scale0):
        starts = np.atleast_2d(np.asarray(starts, dtype=np.float64))
        self.M, self.p = starts.shape
        self.cur = starts.copy()
        self.cur_ll = np.full(self.M, -np.inf)
        self.cur_g = np.zeros_like(starts)
        self.scale = np.full(self.M, float(scale0))
        self.chain = np.zeros((self.M, iters, self.p))
        self.lls = np.zeros((self.M, iters))
        self.acc = np.zeros(self.M, dtype=np.int64)
        self.acc_win = np.zeros(self.M, dtype=np.int64)
        self.fail = np.zeros(self.M, dtype=np.int64)
        self.it = 0
        self.rngs = [np.random.default_rng(s) for s in seeds]

    def save(self, path):
        tmp = path + ".tmp.npz"
        np.savez(tmp, it=self.it, cur=self.cur, cur_ll=self.cur_ll, cur_g=self.cur_g, scale=self.scale,
                 chain=self.chain, lls=self.lls, acc=self.acc, acc_win=self.acc_win, fail=self.fail,
                 rng_states=np.array([r.bit_generator.state for r in self.rngs], dtype=object))
        os.replace(tmp, path)

    def load(self, path):
        ck = np.load(path, allow_pickle=True)
        self.it = int(ck["it"])
        if ck["cur"].shape != self.cur.shape or self.it > self.chain.shape[1]:
            raise ValueError("checkpoint does not match the chains being resumed")
        for k in ("cur", "cur_ll", "cur_g", "scale", "acc", "acc_win", "fail"):
            setattr(self, k, ck[k].copy())
        self.chain[:, : self.it] = ck["chain"][:, : self.it]  # a run may resume with more iterations
        self.lls[:, : self.it] = ck["lls"][:, : self.it]
        for r, st in zip(self.rngs, ck["rng_states"]):
            r.bit_generator.state = st


def _mala_logq(x_to, x_from, g_from, eps):
    """log density (up to a constant) of the MALA proposal x_from -> x_to (identity metric)."""
    mu = x_from + 0.5 * eps * eps * g_from
    d = x_to - mu
    return -0.5 * float(d @ d) / (eps * eps)


def run_chains(obj, starts, iters, burn, seeds, kind="rw", scale0=None, ckpt=None, ckpt_every=100,
               box=(LO, HI), log=None):
    """M chains of random-walk Metropolis (kind 'rw') or MALA (kind 'mala') on x = log(theta)
    with a flat prior on the box, advanced in lockstep: every iteration evaluates the M
    proposals in one batch (obj.batch).  Proposals outside the box are rejected unevaluated,
    failed factorizations are counted and rejected.  During burn-in the step of every chain is
    adapted every 50 iterations towards acceptance 0.3 (rw, codes/19_tlr_mcmc_gpu.py:191-192)
    or 0.574 (mala).  With ckpt the state is written every ckpt_every iterations and a run
    resumes from an existing file; a resumed run is identical to an uninterrupted one."""
    if kind not in ("rw", "mala"):
        raise ValueError("kind must be 'rw' or 'mala'")
    grad = kind == "mala"
    target = 0.3 if kind == "rw" else 0.574
    if scale0 is None:
        scale0 = 0.08 if kind == "rw" else 0.05
    st = ChainState(starts, iters, seeds, scale0)
    if ckpt and os.path.exists(ckpt):
        st.load(ckpt)
        if log:
            log(f"resumed at iteration {st.it}")
    else:
        ll, g = _batch(obj, st.cur, grad)
        if not np.all(np.isfinite(ll)):
            raise RuntimeError("initial state: factorization failed")
        st.cur_ll = ll
        if grad:
            st.cur_g = g
    lo, hi = box
    t_start = time.time()
    for it in range(st.it, iters):
        M = st.M
        prop = np.empty_like(st.cur)
        u = np.empty(M)
        for c in range(M):
            xi = st.rngs[c].standard_normal(st.p)
            if kind == "rw":
                prop[c] = st.cur[c] + st.scale[c] * xi
            else:
                e = st.scale[c]
                prop[c] = st.cur[c] + 0.5 * e * e * st.cur_g[c] + e * xi
            u[c] = st.rngs[c].random()
        inside = np.all((prop > lo) & (prop < hi), axis=1)
        idx = np.nonzero(inside)[0]
        if len(idx):
            ll, g = _batch(obj, prop[idx], grad)
            for q, c in enumerate(idx):
                if not np.isfinite(ll[q]):
                    st.fail[c] += 1
                    continue
                log_a = ll[q] - st.cur_ll[c]
                if grad:
                    e = st.scale[c]
                    log_a += _mala_logq(st.cur[c], prop[c], g[q], e) - _mala_logq(prop[c], st.cur[c], st.cur_g[c], e)
                if np.log(u[c]) < log_a:
                    st.cur[c] = prop[c]
                    st.cur_ll[c] = ll[q]
                    if grad:
                        st.cur_g[c] = g[q]
                    st.acc[c] += 1
                    st.acc_win[c] += 1
        st.chain[:, it] = st.cur
        st.lls[:, it] = st.cur_ll
        st.it = it + 1
        if it < burn and (it + 1) % 50 == 0:
            rate = st.acc_win / 50.0
            st.acc_win[:] = 0
            st.scale *= np.exp(0.5 * (rate - target))
        if log and (it + 1) % 250 == 0:
            log(f"it={it + 1} acc={np.round(st.acc / (it + 1), 2).tolist()} ({time.time() - t_start:.0f}s)")
        if ckpt and (it + 1) % ckpt_every == 0:
            st.save(ckpt)
    return dict(chain=st.chain, lls=st.lls, acceptance=(st.acc / iters).tolist(), failures=st.fail.tolist(),
                scale=st.scale.tolist(), seconds=time.time() - t_start)


# ---------------------------------------------------------------------------------- diagnostics
def _rank_normal_scores(x):
    """Normal scores of the pooled ranks of x (ties share their average rank), with Blom's
    offset: Phi^-1((rank - 3/8) / (S + 1/4)), S = x.size (Vehtari et al. 2021, eq. 14)."""
    from scipy.special import ndtri
    flat = x.ravel()
    order = np.argsort(flat, kind="mergesort")
    srt = flat[order]
    # average rank of each run of equal values: (first + last) / 2 of its 1-based positions
    edges = np.flatnonzero(np.diff(srt) != 0) + 1
    starts = np.concatenate(([0], edges))
    stops = np.concatenate((edges, [srt.size]))
    avg = 0.5 * (starts + 1 + stops)
    ranks = np.empty(flat.size)
    ranks[order] = np.repeat(avg, stops - starts)
    return ndtri((ranks - 0.375) / (flat.size + 0.25)).reshape(x.shape)


def split_rhat_ess(chains):
    """Rank-normalised split R-hat and bulk effective sample size of draws shaped (M chains,
    n draws), following Vehtari, Gelman, Simpson, Carpenter and Buerkner (2021), "Rank-
    normalization, folding, and localization: an improved R-hat", Bayesian Analysis 16:667-718.

    * Every chain is cut into its first and second half (2M sequences of n // 2 draws); all the
      draws are rank-normalised together (_rank_normal_scores).
    * R-hat = sqrt(var+ / W), var+ = (h - 1) / h W + B / h, W the mean within-sequence variance,
      B / h the variance of the sequence means.
    * The autocovariance of every sequence at every lag comes from one zero-padded FFT over the
      sequence axis; rho_t = 1 - (W - mean autocovariance_t) / var+ combines the sequences.
    * ESS = (2M h) / tau with tau = -1 + 2 sum_t P_t over Geyer's (1992, Statistical Science 7:
      473-483) initial monotone sequence of lag pairs P_t = rho_2t + rho_2t+1: cut at the first
      negative pair, then made non-increasing; tau is bounded below by 1 / log10(2M h) as the
      paper does.
    The reference's codes/35_mcmc_multichain_diagnostics.py reports the same two diagnostics for
    its chains."""
    x = np.asarray(chains, dtype=np.float64)
    M, n = x.shape
    h = n // 2
    seq = x[:, :2 * h].reshape(2 * M, h)
    z = _rank_normal_scores(seq)
    m = z.shape[0]
    mu = z.mean(axis=1)
    W = z.var(axis=1, ddof=1).mean()
    var_plus = (h - 1) / h * W + mu.var(ddof=1)
    rhat = float(np.sqrt(var_plus / W))
    dev = z - mu[:, None]
    spec = np.fft.rfft(dev, n=2 * h, axis=1)
    acov = np.fft.irfft(spec * np.conj(spec), n=2 * h, axis=1)[:, :h] / h
    rho = 1.0 - (W - acov.mean(axis=0)) / var_plus
    npair = h // 2
    pairs = rho[0:2 * npair:2] + rho[1:2 * npair:2]
    negative = np.flatnonzero(pairs < 0.0)
    pairs = pairs[:negative[0] if negative.size else npair]
    pairs = np.minimum.accumulate(pairs)
    tau = max(-1.0 + 2.0 * float(pairs.sum()), 1.0 / np.log10(m * h))
    return rhat, float(m * h / tau)


def summarize(chains, burn):
    """Pooled posterior summary on the theta scale of chains shaped (M, iters, 3) on the log scale,
    with per-parameter split R-hat and bulk ESS."""
    th = np.exp(np.asarray(chains)[:, burn:])
    pooled = th.reshape(-1, th.shape[-1])
    rh, es = zip(*[split_rhat_ess(th[:, :, j]) for j in range(th.shape[-1])])
    sd = pooled.std(0, ddof=1)
    return dict(mean=pooled.mean(0).tolist(), sd=sd.tolist(),
                ci95=np.percentile(pooled, [2.5, 97.5], axis=0).T.tolist(), split_rhat=list(rh), bulk_ess=list(es),
                mc_se_of_mean=(sd / np.sqrt(np.maximum(es, 1.0))).tolist(), n_chains=int(th.shape[0]))
