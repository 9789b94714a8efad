"""B200-native adaptive tile-low-rank Gaussian-process log-likelihood.

Drop-in for the TLR log-likelihood path of marysalvana/adaptive-tlr-pilots
(codes/17_tlr_cholesky_pilot.py tlr_loglik and its callers), computed by hand-written sm_100a
CUDA kernels behind the C ABI of include/tlr_b200.h.
"""
from .tlr import (Likelihood, Plan, PlanBatch, TLRFactor, TLRLogLik, dense_loglik, get_kernel,  # noqa: F401
                  get_plan, loglik, loglik_dense_K, make_cov, morton_order, neg_loglik, neg_loglik_tlr,
                  release_plans, set_kernel, skill, tile_bounds, tlr_loglik, tlr_loglik_grad, tlr_predict)

__all__ = ["Likelihood", "Plan", "PlanBatch", "TLRFactor", "TLRLogLik", "dense_loglik", "get_kernel", "get_plan",
           "loglik", "loglik_dense_K", "make_cov", "morton_order", "neg_loglik", "neg_loglik_tlr", "release_plans",
           "set_kernel", "skill", "tile_bounds", "tlr_loglik", "tlr_loglik_grad", "tlr_predict"]
