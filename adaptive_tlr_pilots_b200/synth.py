"""Seeded synthetic Gaussian-process fields, the reference's data protocol on the GPU.

codes/17_tlr_cholesky_pilot.py:313-325: S_all uniform on the unit square, y_all = L z with L the
dense FP64 Cholesky of Sigma(S_all; theta), a random split into N observed and n_pred held-out
sites, Morton order of the observed sites.  The random numbers come from numpy's
default_rng(seed) in the same order as the reference; the dense Cholesky and the product L z run
on the GPU in FP64 (cuSOLVER/cuBLAS through torch), which lets N go past the size where a CPU
LAPACK Cholesky of the (N + n_pred)^2 matrix fails (more than 2^31 entries).  This is data
generation, not part of the likelihood path.
"""
from __future__ import annotations

import numpy as np


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
        K.mul_((3.0 ** 0.5) / rg)
        E = torch.exp(-K)
        K.add_(1.0).mul_(E).mul_(sigma2)
        del E
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
