"""CPU oracle for the adaptive tile-low-rank (TLR) Gaussian-process log-likelihood.

TEST INFRASTRUCTURE ONLY.  This module is a plain NumPy/SciPy restatement of the
reference pipeline (marysalvana/adaptive-tlr-pilots, ``codes/11_tlr_rank_rules.py``
and ``codes/17_tlr_cholesky_pilot.py``).  It exists so that ``tests/``, the smoke check
and the CPU-baseline leg of ``bench.py`` have something independent to compare the
CUDA path with.  The product path (``adaptive_tlr_pilots_b200``) never imports it.

Every function cites the reference lines it follows.  Parity of this restatement with
the reference itself is pinned by ``tests/golden/`` (fixtures generated by importing the
reference, plus the committed result values the reference ships) and checked in
``tests/test_oracle.py``.

Additions that the reference does not have (needed to check the CUDA path):
  * frozen ranks: ``tlr_cholesky(..., rank_log=..., frozen=...)`` records every rank the
    rule picks (initial compression and each recompression) and can replay them at
    another theta, so finite differences see a smooth function;
  * ``singular_tail``: the shared tail/threshold logic, written once.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import LinAlgError, cholesky, solve_triangular
from scipy.linalg import svd as scipy_svd

SQRT3 = np.sqrt(3.0)
LOG2PI = np.log(2.0 * np.pi)


# ----------------------------------------------------------------------------- model
def matern32(h, rng):
    """Matern nu=3/2 correlation (1 + x) exp(-x), x = sqrt(3) h / range.

    Follows codes/11_tlr_rank_rules.py:35-37."""
    x = SQRT3 * h / rng
    return (1.0 + x) * np.exp(-x)


SQRT5 = np.sqrt(5.0)
NU = 1.5  # smoothness of the kernel every covariance below uses (set_kernel)


def matern52(h, rng):
    """Matern nu=5/2 correlation (1 + x + x^2/3) exp(-x), x = sqrt(5) h / range.

    Follows codes/24_screening_stress.py:38-42."""
    x = SQRT5 * h / rng
    return (1.0 + x + x * x / 3.0) * np.exp(-x)


def set_kernel(nu):
    """Select nu = 1.5 or 2.5 for every later covariance: the counterpart of
    codes/24_screening_stress.py:46-47, which patches the kernel of 17 globally."""
    global NU
    if nu not in (1.5, 2.5):
        raise ValueError("nu must be 1.5 or 2.5")
    NU = float(nu)


def matern(h, rng):
    """The selected kernel (set_kernel): matern32 or matern52."""
    return matern52(h, rng) if NU == 2.5 else matern32(h, rng)


def matern_drange(h, rng):
    """d/drange of the selected correlation: x^2 e^{-x} / range (3/2), x^2 (1 + x) e^{-x} / (3 range)
    (5/2).  No counterpart in the reference (it has no gradient code)."""
    if NU == 2.5:
        x = SQRT5 * h / rng
        return x * x * (1.0 + x) * np.exp(-x) / (3.0 * rng)
    x = SQRT3 * h / rng
    return x * x * np.exp(-x) / rng


def morton_order(xy, order=10):
    """Z-order permutation of points in the unit square.

    Coordinates are quantised to ``order`` bits per axis (clip(floor(2^order * c))),
    the x bits go to even and the y bits to odd positions of the key, and the
    permutation is a stable argsort of the key (ties keep input order).
    Follows codes/11_tlr_rank_rules.py:40-53."""
    n = 1 << order
    q = np.clip((xy * n).astype(np.int64), 0, n - 1).astype(np.uint64)

    def interleave_zeros(v):
        out = np.zeros_like(v)
        for bit in range(order):
            out |= ((v >> np.uint64(bit)) & np.uint64(1)) << np.uint64(2 * bit)
        return out

    key = interleave_zeros(q[:, 0]) | (interleave_zeros(q[:, 1]) << np.uint64(1))
    return np.argsort(key, kind="stable")


def pairwise_dist(A, B):
    """Euclidean distances sqrt(max(dx^2 + dy^2, 0)).  codes/11_tlr_rank_rules.py:56-58."""
    d2 = (A[:, None, 0] - B[None, :, 0]) ** 2 + (A[:, None, 1] - B[None, :, 1]) ** 2
    return np.sqrt(np.maximum(d2, 0.0))


def cov_dense(S, theta):
    """Dense covariance sigma2 * M + sigma2 * eta * I.  codes/11_tlr_rank_rules.py:61-65."""
    sigma2, rng, eta = theta
    K = sigma2 * matern(pairwise_dist(S, S), rng)
    K[np.diag_indices_from(K)] += sigma2 * eta
    return K


def tile_bounds(n, b):
    """[(0,b), (b,2b), ..., (.., n)]; the last tile may be short.  codes/11_tlr_rank_rules.py:69-71."""
    edges = list(range(0, n, b)) + [n]
    return [(edges[t], edges[t + 1]) for t in range(len(edges) - 1)]


# ------------------------------------------------------------------------ rank rule
def singular_tail(s):
    """tail[r] = ||T - T_r||_F for r = 0..len(s), with tail[len(s)] = 0.

    Summed from the smallest singular value up, as codes/17_tlr_cholesky_pilot.py:113."""
    return np.append(np.sqrt(np.cumsum(s[::-1] ** 2)[::-1]), 0.0)


def choose_rank(s, rule, thr_rel, thr_abs):
    """Smallest r with tail[r] <= threshold; threshold is thr_rel*||s||_2 for 'fixed' and
    thr_abs for 'adaptive'.  codes/17_tlr_cholesky_pilot.py:113-115 (same rule at 130-132,
    codes/11_tlr_rank_rules.py:92-98)."""
    tail = singular_tail(s)
    thr = thr_rel * np.sqrt((s ** 2).sum()) if rule == "fixed" else thr_abs
    return int(np.argmax(tail <= thr)), tail


def _svd(T, full_matrices=False):
    # gesdd first, gesvd when it does not converge: codes/17_tlr_cholesky_pilot.py:109-112
    try:
        return np.linalg.svd(T, full_matrices=full_matrices)
    except np.linalg.LinAlgError:
        return scipy_svd(T, full_matrices=full_matrices, lapack_driver="gesvd")


def truncate_svd(T, rule, thr_rel, thr_abs, rank=None):
    """Rank-r truncation of a dense tile: returns (U*s, V, tail[r], r).

    codes/17_tlr_cholesky_pilot.py:107-116.  ``rank`` overrides the rule (frozen ranks)."""
    U, s, Vt = _svd(T)
    r, tail = choose_rank(s, rule, thr_rel, thr_abs)
    if rank is not None:
        r = int(rank)
    return U[:, :r] * s[:r], Vt[:r].T, float(tail[r]), r


def recompress(U, V, rule, thr_rel, thr_abs, rank=None):
    """Recompress U V^T: QR(U), QR(V), SVD of the k x k core R_u R_v^T, same rule.

    codes/17_tlr_cholesky_pilot.py:119-133.  ``rank`` overrides the rule."""
    if U.shape[1] == 0:
        return U, V, 0.0, 0
    Qu, Ru = np.linalg.qr(U)
    Qv, Rv = np.linalg.qr(V)
    Uw, s, Vwt = _svd(Ru @ Rv.T, full_matrices=True)
    r, tail = choose_rank(s, rule, thr_rel, thr_abs)
    if rank is not None:
        r = int(rank)
    return Qu @ (Uw[:, :r] * s[:r]), Qv @ Vwt[:r].T, float(tail[r]), r


def thresholds(n, b, theta, rule, value):
    """(thr_rel, thr_abs): fixed -> eps; adaptive -> tau * b * sigma2 * eta / N.

    codes/17_tlr_cholesky_pilot.py:143-150 (b is the largest tile size)."""
    sigma2, _, eta = theta
    thr_rel = value if rule == "fixed" else None
    thr_abs = value * b * sigma2 * eta / n if rule == "adaptive" else None
    return thr_rel, thr_abs


# ------------------------------------------------------- storage precision (rule 'mixed')
STORAGE_BITS = (8, 16, 32, 64)


def round_fp8(x):
    """The reference's simulated FP8 (E4M3-like) rounding: |x| = m 2^e with e = floor(log2|x|)
    clipped to [-9, 8], m rounded to 3 fraction bits (half to even), values above 448 set to 448,
    zeros kept.  codes/17_tlr_cholesky_pilot.py:41-55 (the p = 8 branch)."""
    x = np.asarray(x, dtype=np.float64)
    a = np.abs(x)
    out = np.zeros_like(x)
    nz = a > 0
    e = np.clip(np.floor(np.log2(a[nz])), -9, 8)
    v = np.round(a[nz] / 2.0 ** e * 8.0) / 8.0 * 2.0 ** e
    out[nz] = np.sign(x[nz]) * np.minimum(v, 448.0)
    return out


def round_bits(x, p):
    """x rounded to p-bit storage: 64 unchanged, 32 / 16 through numpy float32 / float16 casts,
    8 through round_fp8.  codes/17_tlr_cholesky_pilot.py:41-55."""
    if p == 64:
        return x
    if p == 32:
        return x.astype(np.float32).astype(np.float64)
    if p == 16:
        return x.astype(np.float16).astype(np.float64)
    return round_fp8(x)


def store_factor(U, p):
    """A factor as stored in p bits: for p < 32 scaled so its largest magnitude is half the
    format's largest value (224 for FP8, 32752 for FP16) before rounding, unscaled after.
    codes/17_tlr_cholesky_pilot.py:58-66."""
    if p == 64 or U.size == 0:
        return U
    top = np.abs(U).max()
    if top == 0:
        return U
    if p == 32:
        return round_bits(U, 32)
    scale = (224.0 if p == 8 else 32752.0) / top
    return round_bits(U * scale, p) / scale


def round_pair(U, V, budget):
    """(U', V', p): the pair stored in the fewest bits p in (8, 16, 32) whose rounding error
    ||U V^T - U' V'^T||_F is at most `budget`, else unchanged with p = 64.
    codes/17_tlr_cholesky_pilot.py:69-82."""
    if U.shape[1] == 0:
        return U, V, 64
    T = U @ V.T
    for p in STORAGE_BITS[:-1]:
        Ur, Vr = store_factor(U, p), store_factor(V, p)
        if np.linalg.norm(T - Ur @ Vr.T) <= budget:
            return Ur, Vr, p
    return U, V, 64


# ------------------------------------------------------------------ TLR Cholesky
def tlr_cholesky(S, theta, bounds, rule, value, rank_log=None, frozen=None, on_stage=None):
    """Right-looking TLR Cholesky of Sigma(theta) without forming Sigma.

    Returns (L_diag, L_off, info) or (None, None, info) when a diagonal tile is not
    positive definite.  L_off[(i, j)] = (U, V), L_ij ~ U V^T, i > j, in the insertion
    order of the reference (for k, for i > k).  codes/17_tlr_cholesky_pilot.py:137-215
    for rules 'fixed' and 'adaptive'.

    rank_log: optional dict, filled with {('init', i, j): r, ('rc', k, i, j): r}, and under rule
              'mixed' with the storage bits of every rounding: ('init_bits', i, j), ('trsm_bits', i, k),
              ('rc_bits', k, i, j).
    frozen:   optional dict of the same form; its ranks replace the rule's choice.
    on_stage: optional callable, called with ("compress", i) after tile row i is generated and
              compressed and with ("factor", k) after factorization step k (for stage timings).
    """
    if rule not in ("fixed", "adaptive", "mixed"):
        raise ValueError(f"rule must be 'fixed', 'adaptive' or 'mixed', got {rule!r}")
    # rule 'mixed' (17:33-40, 145-148): the adaptive ranks, every stored pair rounded by round_pair
    mixed = rule == "mixed"
    if mixed:
        rule = "adaptive"
    prec = {}  # (i, j) -> bits of the stored factor tile (rule 'mixed')
    n = S.shape[0]
    nB = len(bounds)
    b = max(e - s for s, e in bounds)
    sigma2, rng, eta = theta
    nugget = sigma2 * eta
    thr_rel, thr_abs = thresholds(n, b, theta, rule, value)

    def pick(key):
        return None if frozen is None else frozen[key]

    # tile generation + initial compression: 17:151-167
    A_diag = []
    A_off = {}
    stored0 = 0
    for i, (i0, i1) in enumerate(bounds):
        D = sigma2 * matern(pairwise_dist(S[i0:i1], S[i0:i1]), rng)
        D[np.diag_indices_from(D)] += nugget
        A_diag.append(D)
        stored0 += (i1 - i0) ** 2
        for j, (j0, j1) in enumerate(bounds[:i]):
            T = sigma2 * matern(pairwise_dist(S[i0:i1], S[j0:j1]), rng)
            U, V, tail, r = truncate_svd(T, rule, thr_rel, thr_abs, pick(("init", i, j)))
            if rank_log is not None:
                rank_log[("init", i, j)] = r
            if mixed:  # 17:163-164
                U, V, bits = round_pair(U, V, thr_abs - tail)
                if rank_log is not None:
                    rank_log[("init_bits", i, j)] = bits
            A_off[(i, j)] = (U, V)
            stored0 += 2 * r * max(i1 - i0, j1 - j0)
        if on_stage is not None:
            on_stage(("compress", i))
    sigma_ranks = [u.shape[1] for u, _ in A_off.values()]
    info = dict(stored_sigma=int(stored0), max_rank_sigma=max(sigma_ranks) if sigma_ranks else 0,
                sigma_ranks=sigma_ranks)

    L_diag = [None] * nB
    L_off = {}
    for k in range(nB):
        # diagonal POTRF: 17:171-177
        try:
            Lkk = cholesky(A_diag[k], lower=True, check_finite=False)
        except LinAlgError:
            info.update(completed=False, failed_at=k)
            return None, None, info
        L_diag[k] = Lkk
        # panel TRSM, V <- L_kk^{-1} V: 17:178-185
        for i in range(k + 1, nB):
            U, V = A_off.pop((i, k))
            if U.shape[1]:
                V = solve_triangular(Lkk, V, lower=True, check_finite=False)
            if mixed:  # 17:183-184
                U, V, prec[(i, k)] = round_pair(U, V, thr_abs)
                if rank_log is not None:
                    rank_log[("trsm_bits", i, k)] = prec[(i, k)]
            L_off[(i, k)] = (U, V)
        # trailing update A_ij -= L_ik L_jk^T with recompression: 17:186-205
        for i in range(k + 1, nB):
            Ui, Vi = L_off[(i, k)]
            if Ui.shape[1] == 0:
                continue
            for j in range(k + 1, i + 1):
                Uj, Vj = L_off[(j, k)]
                if Uj.shape[1] == 0:
                    continue
                W = Vi.T @ Vj
                if i == j:
                    A_diag[i] -= (Ui @ W) @ Ui.T
                else:
                    Uij, Vij = A_off[(i, j)]
                    Ur, Vr, tail, r = recompress(np.hstack([Uij, -(Ui @ W)]), np.hstack([Vij, Uj]),
                                                 rule, thr_rel, thr_abs, pick(("rc", k, i, j)))
                    if rank_log is not None:
                        rank_log[("rc", k, i, j)] = r
                    if mixed:  # 17:203-204
                        Ur, Vr, bits = round_pair(Ur, Vr, thr_abs - tail)
                        if rank_log is not None:
                            rank_log[("rc_bits", k, i, j)] = bits
                    A_off[(i, j)] = (Ur, Vr)
        if on_stage is not None:
            on_stage(("factor", k))
    # storage statistics: 17:206-209
    ranks = [u.shape[1] for u, _ in L_off.values()]
    stored = sum(d.shape[0] ** 2 for d in L_diag) + sum(2 * u.shape[1] * u.shape[0] for u, _ in L_off.values())
    info.update(completed=True, stored_factor=int(stored),
                mean_rank_factor=float(np.mean(ranks)) if ranks else 0.0,
                max_rank_factor=int(max(ranks)) if ranks else 0, factor_ranks=ranks)
    if mixed:  # bytes of the stored factor and the precision mix: 17:210-214
        byt = sum(d.shape[0] ** 2 * 8 for d in L_diag) + sum(2 * u.shape[1] * u.shape[0] * prec[key] // 8
                                                             for key, (u, _) in L_off.items())
        dense = n * (n + 1) // 2 * 8
        info.update(stored_factor_bytes=int(byt), dense_factor_bytes=int(dense), factor_bytes_frac=byt / dense,
                    precision_mix_factor_tiles={q: int(sum(1 for key in L_off if prec[key] == q)) for q in STORAGE_BITS},
                    factor_prec=[prec[key] for key in L_off])
    return L_diag, L_off, info


def tlr_matvec_L(L_diag, L_off, bounds, Z):
    """Y = L Z for the tile factor.  codes/17_tlr_cholesky_pilot.py:218-227."""
    Y = np.zeros_like(Z)
    for k, (k0, k1) in enumerate(bounds):
        Y[k0:k1] = L_diag[k] @ Z[k0:k1]
        for j, (j0, j1) in enumerate(bounds[:k]):
            U, V = L_off[(k, j)]
            if U.shape[1]:
                Y[k0:k1] += U @ (V.T @ Z[j0:j1])
    return Y


def tlr_forward(L_diag, L_off, bounds, B):
    """Solve L Z = B tile by tile.  codes/17_tlr_cholesky_pilot.py:230-240."""
    Z = np.zeros_like(B)
    for k, (k0, k1) in enumerate(bounds):
        rhs = B[k0:k1].copy()
        for j, (j0, j1) in enumerate(bounds[:k]):
            U, V = L_off[(k, j)]
            if U.shape[1]:
                rhs -= U @ (V.T @ Z[j0:j1])
        Z[k0:k1] = solve_triangular(L_diag[k], rhs, lower=True, check_finite=False)
    return Z


def tlr_backward(L_diag, L_off, bounds, Z):
    """Solve L^T X = Z tile by tile.  codes/17_tlr_cholesky_pilot.py:243-256."""
    nB = len(bounds)
    X = np.zeros_like(Z)
    for k in range(nB - 1, -1, -1):
        k0, k1 = bounds[k]
        rhs = Z[k0:k1].copy()
        for i in range(k + 1, nB):
            i0, i1 = bounds[i]
            U, V = L_off[(i, k)]
            if U.shape[1]:
                rhs -= V @ (U.T @ X[i0:i1])
        X[k0:k1] = solve_triangular(L_diag[k], rhs, lower=True, trans="T", check_finite=False)
    return X


def tlr_predict(S, y, Sp, theta, bounds, fac):
    """Kriging mean and standard deviation with the tile factor.  codes/17_tlr_cholesky_pilot.py:269-276."""
    L_diag, L_off = fac
    Kp = theta[0] * matern(pairwise_dist(Sp, S), theta[1])
    alpha = tlr_backward(L_diag, L_off, bounds, tlr_forward(L_diag, L_off, bounds, y[:, None]))[:, 0]
    mu = Kp @ alpha
    W = tlr_forward(L_diag, L_off, bounds, Kp.T)
    var = theta[0] * (1 + theta[2]) - (W ** 2).sum(0)
    return mu, np.sqrt(np.maximum(var, 1e-12))


def skill(yp, mu, sig):
    """RMSE, Gaussian CRPS and 90% coverage.  codes/11_tlr_rank_rules.py:142-146, 162-165."""
    from scipy.special import erf
    z = (yp - mu) / sig
    pdf = np.exp(-0.5 * z ** 2) / np.sqrt(2 * np.pi)
    cdf = 0.5 * (1 + erf(z / np.sqrt(2)))
    crps = float((sig * (z * (2 * cdf - 1) + 2 * pdf - 1 / np.sqrt(np.pi))).mean())
    return dict(rmse=float(np.sqrt(((yp - mu) ** 2).mean())), crps=crps, cover90=float((np.abs(z) <= 1.6448536).mean()))


def tlr_loglik(S, y, theta, bounds, rule, value, rank_log=None, frozen=None, on_stage=None):
    """(loglik | None, (L_diag, L_off) | None, info).

    l = -1/2 (z^T z + 2 sum log diag L_kk + N log 2 pi), z = L^{-1} y.
    codes/17_tlr_cholesky_pilot.py:259-266."""
    L_diag, L_off, info = tlr_cholesky(S, theta, bounds, rule, value, rank_log=rank_log, frozen=frozen,
                                       on_stage=on_stage)
    if L_diag is None:
        return None, None, info
    z = tlr_forward(L_diag, L_off, bounds, y[:, None])[:, 0]
    logdet = 2.0 * sum(np.log(np.diag(d)).sum() for d in L_diag)
    ll = -0.5 * (z @ z + logdet + len(y) * LOG2PI)
    info.update(logdet=float(logdet), quad=float(z @ z))
    return float(ll), (L_diag, L_off), info


def matern32_dtheta(S, bounds, theta, i, j):
    """(dSigma/dsigma2, dSigma/drange, dSigma/deta) of tile (i, j) for the selected kernel:
    Sigma/sigma2 (+ eta I on the diagonal), sigma2 dk/drange (matern_drange), and sigma2 I on the
    diagonal.  No counterpart in the reference (it has no gradient code)."""
    sigma2, rng, eta = theta
    (i0, i1), (j0, j1) = bounds[i], bounds[j]
    h = pairwise_dist(S[i0:i1], S[j0:j1])
    ds = matern(h, rng)
    dr = sigma2 * matern_drange(h, rng)
    de = np.zeros_like(ds)
    if i == j:
        ds[np.diag_indices_from(ds)] += eta
        de[np.diag_indices_from(de)] = sigma2
    return ds, dr, de


def tlr_loglik_grad(S, y, theta, bounds, rule, value):
    """Log-likelihood and its gradient in (sigma2, range, eta) through the TLR factor.

    With Sigma_t = L L^T the TLR approximation (ranks as chosen at theta, frozen), the gradient is
        dl/dtheta = 1/2 alpha^T dSigma alpha - 1/2 tr(Z dSigma),   alpha = Sigma_t^{-1} y,
    Z = Sigma_t^{-1}, dSigma the derivative of the covariance tiles (regenerated from the sites).
    Z's tiles come from the selected-inversion (Takahashi) recurrence on the tile factor, which
    is the blocked Cholesky adjoint with every truncation passed through unchanged:
        Z_ik = -(sum_{j>k} Z_ij L_jk) L_kk^{-1}                      (i > k)
        Z_kk = (L_kk^{-T} - sum_{j>k} Z_jk^T L_jk) L_kk^{-1}.
    As the rank rule tightens this tends to the dense gradient; at the reference's adaptive
    tau = 0.9 it differs from finite differences of the frozen-rank TLR log-likelihood by
    O(truncation).  No counterpart in the reference.  Returns (ll | None, grad | None, info)."""
    ll, fac, info = tlr_loglik(S, y, theta, bounds, rule, value)
    if ll is None:
        return None, None, info
    Ld, Lo = fac
    nB = len(bounds)
    z = tlr_forward(Ld, Lo, bounds, y[:, None])
    alpha = tlr_backward(Ld, Lo, bounds, z)[:, 0]
    Z = {}
    for k in range(nB - 1, -1, -1):
        js = list(range(k + 1, nB))
        Lkk = Ld[k]
        Li = solve_triangular(Lkk, np.eye(Lkk.shape[0]), lower=True, check_finite=False)
        if js:
            Vp = Li.T @ np.hstack([Lo[(j, k)][1] for j in js])
            for i in js:
                Ci = np.hstack([(Z[(i, j)] if i >= j else Z[(j, i)].T) @ Lo[(j, k)][0] for j in js])
                Z[(i, k)] = -Ci @ Vp.T
            acc = np.zeros_like(Lkk)
            for j in js:
                U, V = Lo[(j, k)]
                acc += (Z[(j, k)].T @ U) @ V.T
            Z[(k, k)] = (Li.T - acc) @ Li
        else:
            Z[(k, k)] = Li.T @ Li
    g = np.zeros(3)
    for i in range(nB):
        i0, i1 = bounds[i]
        for j in range(i + 1):
            j0, j1 = bounds[j]
            w = 1.0 if i == j else 2.0
            Sbar = 0.5 * np.outer(alpha[i0:i1], alpha[j0:j1]) - 0.5 * Z[(i, j)]
            for a, dT in enumerate(matern32_dtheta(S, bounds, theta, i, j)):
                g[a] += w * np.sum(Sbar * dT)
    return ll, g, info


def neg_loglik_tlr(logth, S, y, bounds, rule, value, trace):
    """Optimizer wrapper: 1e12 on a failed factorization.  codes/17_tlr_cholesky_pilot.py:279-290."""
    theta = np.exp(logth)
    trace["evals"] += 1
    if rule == "dense":
        ll, _ = loglik_dense(cov_dense(S, theta), y)
    else:
        ll, _, _ = tlr_loglik(S, y, theta, bounds, rule, value)
    if ll is None:
        trace["failures"] += 1
        return 1e12
    return -ll


# -------------------------------------------------------------------------- dense oracle
def loglik_dense(K, y):
    """Dense FP64 log-likelihood by Cholesky; (None, None) when K is not PD.

    codes/11_tlr_rank_rules.py:112-120."""
    try:
        c = cholesky(K, lower=True, check_finite=False)
    except LinAlgError:
        return None, None
    z = solve_triangular(c, y, lower=True, check_finite=False)
    logdet = 2.0 * np.log(np.diag(c)).sum()
    return float(-0.5 * (z @ z + logdet + len(y) * LOG2PI)), c


def dense_loglik_and_grad(S, y, theta):
    """Dense FP64 log-likelihood and its gradient in (sigma2, range, eta).

    dl/dtheta = 1/2 alpha^T dK alpha - 1/2 tr(K^{-1} dK), alpha = K^{-1} y, with
    dK/dsigma2 = K/sigma2, dK/drange = sigma2 dk/drange of the selected kernel (matern_drange),
    dK/deta = sigma2 I.  No counterpart in the reference (it has no gradient code)."""
    sigma2, rng, eta = theta
    H = pairwise_dist(S, S)
    M = matern(H, rng)
    K = sigma2 * M
    K[np.diag_indices_from(K)] += sigma2 * eta
    c = cholesky(K, lower=True, check_finite=False)
    z = solve_triangular(c, y, lower=True, check_finite=False)
    alpha = solve_triangular(c, z, lower=True, trans="T", check_finite=False)
    Ci = solve_triangular(c, np.eye(len(y)), lower=True, check_finite=False)
    Kinv = Ci.T @ Ci
    ll = -0.5 * (z @ z + 2.0 * np.log(np.diag(c)).sum() + len(y) * LOG2PI)
    dKs = M + eta * np.eye(len(y))
    dKr = sigma2 * matern_drange(H, rng)
    grads = []
    for dK in (dKs, dKr, None):
        if dK is None:
            grads.append(0.5 * sigma2 * (alpha @ alpha) - 0.5 * sigma2 * np.trace(Kinv))
        else:
            grads.append(0.5 * alpha @ dK @ alpha - 0.5 * np.sum(Kinv * dK))
    return float(ll), np.array(grads)


# ---------------------------------------------------------- assembled-matrix rank rule
def truncate_tiles(K, bounds, rule, value, m_theta):
    """Truncate every off-diagonal tile of an assembled K in place.

    Returns (stored, max_rel, max_abs, ||Delta||_F, ranks).  codes/11_tlr_rank_rules.py:74-108."""
    n = K.shape[0]
    b = max(e - s for s, e in bounds)
    stored = sum((e - s) ** 2 for s, e in bounds)
    emax = value * b * m_theta / n
    ranks, max_rel, max_abs, fro2 = [], 0.0, 0.0, 0.0
    for i, (i0, i1) in enumerate(bounds):
        for j, (j0, j1) in enumerate(bounds[:i]):
            T = K[i0:i1, j0:j1]
            U, s, Vt = _svd(T)
            r, tail = choose_rank(s, rule, value, emax)
            Tr = (U[:, :r] * s[:r]) @ Vt[:r] if r > 0 else np.zeros_like(T)
            err = tail[r]
            K[i0:i1, j0:j1] = Tr
            K[j0:j1, i0:i1] = Tr.T
            stored += 2 * r * max(i1 - i0, j1 - j0)
            ranks.append(r)
            fro2 += 2 * err ** 2
            max_abs = max(max_abs, err)
            max_rel = max(max_rel, err / max(np.sqrt((s ** 2).sum()), 1e-300))
    return stored, max_rel, max_abs, float(np.sqrt(fro2)), ranks


# ------------------------------------------------------------------ data protocol
def simulate_field(n, theta=(1.0, 0.3, 0.05), n_pred=300, seed=20261020):
    """Seeded synthetic field: uniform sites, y = L z with L the dense FP64 Cholesky of
    Sigma(S_all), a random split into n observed / n_pred held out, Morton order of the
    observed sites.  codes/17_tlr_cholesky_pilot.py:313-325.

    Returns (S, y, Sp, yp) with S, y Morton-ordered."""
    rng = np.random.default_rng(seed)
    theta = np.asarray(theta, float)
    n_tot = n + n_pred
    S_all = rng.random((n_tot, 2))
    L = np.linalg.cholesky(cov_dense(S_all, theta))
    y_all = L @ rng.standard_normal(n_tot)
    del L
    perm = rng.permutation(n_tot)
    obs, hold = perm[:n], perm[n:]
    S, y, Sp, yp = S_all[obs], y_all[obs], S_all[hold], y_all[hold]
    order = morton_order(S)
    return S[order], y[order], Sp, yp


def simulate_sites(n, n_pred=300, seed=20261020):
    """Sites only (no field), Morton-ordered, drawn in the same order as simulate_field
    (S_all first, then the permutation is drawn after the field's normals)."""
    rng = np.random.default_rng(seed)
    S_all = rng.random((n + n_pred, 2))
    rng.standard_normal(n + n_pred)
    perm = rng.permutation(n + n_pred)
    S = S_all[perm[:n]]
    return S[morton_order(S)]
