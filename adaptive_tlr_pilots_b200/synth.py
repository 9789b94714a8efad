"""Seeded synthetic Gaussian-process fields, the reference's data protocol on the GPU.

codes/17_tlr_cholesky_pilot.py:313-325: S_all uniform on the unit square, y_all = L z with L the
dense FP64 Cholesky of Sigma(S_all; theta), a random split into N observed and n_pred held-out
sites, Morton order of the observed sites (the kernel chosen by tlr.set_kernel, as the reference's
sweeps simulate with the kernel they patch in, codes/24_screening_stress.py:58-59).  The random numbers come from numpy's
default_rng(seed) in the same order as the reference; the dense Cholesky and the product L z run
on the GPU in FP64 (cuSOLVER/cuBLAS through torch), which lets N go past the size where a CPU
LAPACK Cholesky of the (N + n_pred)^2 matrix fails (more than 2^31 entries).  This is data
generation, not part of the likelihood path.
"""
from __future__ import annotations

import numpy as np


def _matern_inplace(K, rg, sigma2):
    """K (distances) <- sigma2 k(K / range) in place for the kernel chosen by tlr.set_kernel."""
    import torch

    from .tlr import get_kernel
    if get_kernel() == 2.5:  # (1 + x + x^2 / 3) e^{-x}, x = sqrt(5) h / range (24:38-42)
        K.mul_((5.0 ** 0.5) / rg)
        E = torch.exp(-K)
        K.mul_(K.div(3.0).add_(1.0)).add_(1.0).mul_(E).mul_(sigma2)
    else:
        K.mul_((3.0 ** 0.5) / rg)
        E = torch.exp(-K)
        K.add_(1.0).mul_(E).mul_(sigma2)
    del E


def simulate_field(n, theta=(1.0, 0.3, 0.05), n_pred=300, seed=20261020, device=0, order_fn=None):
    """Returns (S, y, Sp, yp), S and y in Morton order.  order_fn(S) -> permutation defaults to
    the GPU Morton order of this package."""
    import torch

    from .tlr import morton_order
    if order_fn is None:
        def order_fn(P):
            return morton_order(P, device=device)
    rng = np.random.default_rng(seed)
    n_tot = n + n_pred
    S_all = rng.random((n_tot, 2))
    z = rng.standard_normal(n_tot)
    perm = rng.permutation(n_tot)
    dev = torch.device("cuda", device)
    sigma2, rg, eta = [float(v) for v in theta]
    with torch.no_grad():
        St = torch.as_tensor(S_all, device=dev)
        K = torch.cdist(St, St)
        _matern_inplace(K, rg, sigma2)
        K.diagonal().add_(sigma2 * eta)
        L, info = torch.linalg.cholesky_ex(K)
        del K
        if int(info.item()) != 0:
            raise RuntimeError("simulation covariance is not positive definite")
        y_all = (L @ torch.as_tensor(z, device=dev)).cpu().numpy()
        del L
        torch.cuda.empty_cache()
    obs, hold = perm[:n], perm[n:]
    S, y, Sp, yp = S_all[obs], y_all[obs], S_all[hold], y_all[hold]
    order = order_fn(S)
    return S[order], y[order], Sp, yp


def dense_loglik_gpu(S, y, theta, device=0):
    """Dense FP64 log-likelihood by a GPU Cholesky (the dense oracle at sizes where the CPU one
    fails); None when not positive definite."""
    from .tlr import dense_loglik
    return dense_loglik(S, y, theta, device=device)


def dense_loglik_grad_gpu(S, y, theta, device=0, chunk=4096):
    """Dense FP64 log-likelihood and its gradient in (sigma2, range, eta) on the GPU
    (cuSOLVER Cholesky and inverse through torch; dSigma in row blocks): the dense oracle for the
    gradient at sizes where a CPU Cholesky fails.  Returns (ll, grad) or (None, None)."""
    import torch

    from .tlr import get_kernel
    dev = torch.device("cuda", device)
    sigma2, rg, eta = [float(v) for v in theta]
    with torch.no_grad():
        St = torch.as_tensor(np.asarray(S, dtype=np.float64), device=dev)
        yt = torch.as_tensor(np.asarray(y, dtype=np.float64), device=dev)
        n = St.shape[0]
        K = torch.cdist(St, St)
        _matern_inplace(K, rg, sigma2)
        K.diagonal().add_(sigma2 * eta)
        L, info = torch.linalg.cholesky_ex(K)
        del K
        if int(info.item()) != 0:
            return None, None
        z = torch.linalg.solve_triangular(L, yt[:, None], upper=False)
        ll = float(-0.5 * ((z * z).sum() + 2.0 * torch.log(torch.diagonal(L)).sum() + n * np.log(2 * np.pi)))
        alpha = torch.cholesky_solve(yt[:, None], L)[:, 0]
        Kinv = torch.cholesky_inverse(L)
        del L
        g = np.zeros(3)
        for r0 in range(0, n, chunk):
            r1 = min(n, r0 + chunk)
            nu5 = get_kernel() == 2.5
            x = torch.cdist(St[r0:r1], St) * (((5.0 if nu5 else 3.0) ** 0.5) / rg)
            e = torch.exp(-x)
            W = 0.5 * (alpha[r0:r1, None] * alpha[None, :] - Kinv[r0:r1])
            if nu5:
                g[0] += float(((1.0 + x + x * x / 3.0) * e * W).sum())
                g[1] += float((sigma2 * x * x * (1.0 + x) / 3.0 * e / rg * W).sum())
            else:
                g[0] += float(((1.0 + x) * e * W).sum())
                g[1] += float((sigma2 * x * x * e / rg * W).sum())
            del x, e
            idx = torch.arange(r0, r1, device=dev)
            wd = W[idx - r0, idx]
            g[0] += float(eta * wd.sum())
            g[2] += float(sigma2 * wd.sum())
        del Kinv
        torch.cuda.empty_cache()
    return ll, g


def simulate_field_tlr(n, theta=(1.0, 0.3, 0.05), b=1000, tau=0.02, n_pred=300, seed=20261020, device=0):
    """Field for sizes where no dense factor fits (codes/17_tlr_cholesky_pilot.py:326-339, --sim tlr):
    sites and split as the dense protocol, then y = L z with L the TLR factor of Sigma(S; theta)
    at the tight adaptive budget tau = 0.02 (tlr_factor_matvec on the device), and held-out values
    from the TLR predictive mean plus noise.  Returns (S, y, Sp, yp, info) with S, y Morton-ordered."""
    import torch

    from .tlr import Plan, TLRFactor, morton_order, tlr_predict, tile_bounds
    rng = np.random.default_rng(seed)
    n_tot = n + n_pred
    S_all = rng.random((n_tot, 2))
    perm = rng.permutation(n_tot)
    obs, hold = perm[:n], perm[n:]
    S, Sp = S_all[obs], S_all[hold]
    S = S[morton_order(S, device=device)]
    plan = Plan(n, b, cap=128, device=device)  # tau = 0.02 keeps ranks up to ~100 near the diagonal
    plan.set_data(S, np.zeros(n))
    ev = plan.evaluate(theta, "adaptive", tau)
    if ev.status != 0:
        plan.close()
        raise RuntimeError("simulation factor did not complete")
    z = rng.standard_normal(n_tot)
    y = plan.matvec_L(torch.from_numpy(z[:n])).cpu().numpy()
    plan.set_data(S, y)  # the factor does not depend on y; the solves below use it as is
    fac = TLRFactor(plan)
    mu_p, sd_p = tlr_predict(S, y, Sp, theta, tile_bounds(n, b), fac)
    yp = mu_p + sd_p * z[n:]
    info = dict(ev.info, factor_fraction_of_dense=ev.info["stored_factor"] / (n * (n + 1) / 2))
    plan.close()
    return S, y, Sp, yp, info
