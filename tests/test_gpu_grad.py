"""Device gradient (backward kernels) against the oracle's gradient of the same formula, and the
documented comparisons with finite differences and the dense FP64 gradient."""
import json
import os

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


@pytest.mark.parametrize("case,b,theta,rule,value", [
    ("n1030_b100", 100, (1.0, 0.3, 0.05), "adaptive", 0.9),
    ("n1030_b100", 100, (1.0, 0.3, 0.05), "fixed", 1e-6),
    ("n1500_b250_s2.5_r0.1", 250, (2.5, 0.1, 0.2), "adaptive", 0.5),
    ("n2000_b200_r1.0_e0.005", 200, (1.0, 1.0, 0.005), "adaptive", 0.9),
])
def test_grad_matches_oracle(tlr, case, b, theta, rule, value):
    d = np.load(os.path.join(GOLD, case + "_data.npz"))
    S, y = d["S"], d["y"]
    bounds = tlr.tile_bounds(len(y), b)
    ll, g, info = tlr.tlr_loglik_grad(S, y, theta, bounds, rule, value)
    ll_o, g_o, info_o = O.tlr_loglik_grad(S, y, theta, bounds, rule, value)
    assert abs(ll - ll_o) <= 1e-10 * abs(ll_o)
    np.testing.assert_allclose(g, g_o, rtol=1e-8, atol=1e-8 * np.abs(g_o).max())


def test_grad_close_to_dense_and_fd_for_tight_rule(tlr):
    """With a tight rule (fixed eps = 1e-8) the TLR gradient is within 1e-5 (relative, 2-norm) of
    the dense FP64 gradient and of central differences of the frozen-rank TLR log-likelihood."""
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    S, y = d["S"], d["y"]
    theta = np.array([1.0, 0.3, 0.05])
    bounds = tlr.tile_bounds(len(y), 100)
    ll, g, info = tlr.tlr_loglik_grad(S, y, theta, bounds, "fixed", 1e-8)
    _, gd = O.dense_loglik_and_grad(S, y, theta)
    assert np.linalg.norm(g - gd) <= 1e-5 * np.linalg.norm(gd)
    log = {}
    O.tlr_loglik(S, y, theta, bounds, "fixed", 1e-8, rank_log=log)
    fd = np.zeros(3)
    for a in range(3):
        h = 1e-5 * theta[a]
        tp, tm = theta.copy(), theta.copy()
        tp[a] += h
        tm[a] -= h
        fd[a] = (O.tlr_loglik(S, y, tp, bounds, "fixed", 1e-8, frozen=log)[0]
                 - O.tlr_loglik(S, y, tm, bounds, "fixed", 1e-8, frozen=log)[0]) / (2 * h)
    assert np.linalg.norm(g - fd) <= 1e-5 * np.linalg.norm(fd)


def test_autograd_function(tlr):
    import torch
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    plan = tlr.get_plan(1030, 100)
    plan.set_data(d["S"], d["y"])
    theta = torch.tensor([1.0, 0.3, 0.05], dtype=torch.float64, requires_grad=True)
    ll = tlr.TLRLogLik.apply(theta, plan, "adaptive", 0.9)
    ll.backward()
    _, g_o, _ = O.tlr_loglik_grad(d["S"], d["y"], (1.0, 0.3, 0.05), O.tile_bounds(1030, 100), "adaptive", 0.9)
    np.testing.assert_allclose(theta.grad.numpy(), g_o, rtol=1e-8)


@pytest.mark.parametrize("case,b,rule,value", [
    ("n1030_b100", 100, "adaptive", 0.9),
    ("n4000_b250", 250, "adaptive", 0.9),
])
def test_mixed_gradient_close_to_fp64(tlr, case, b, rule, value):
    """Tensor-core 3xTF32 backward: gradient within 1e-4 (relative, 2-norm) of the FP64 backward."""
    d = np.load(os.path.join(GOLD, case + "_data.npz"))
    n = len(d["y"])
    p64 = tlr.Plan(n, b)
    p64.set_data(d["S"], d["y"])
    e64 = p64.evaluate((1.0, 0.3, 0.05), rule, value, grad=True)
    pmx = tlr.Plan(n, b)
    pmx.set_precision("mixed")
    pmx.set_data(d["S"], d["y"])
    emx = pmx.evaluate((1.0, 0.3, 0.05), rule, value, grad=True)
    assert abs(emx.loglik - e64.loglik) <= 1e-2
    assert np.linalg.norm(emx.grad - e64.grad) <= 1e-4 * np.linalg.norm(e64.grad), (emx.grad, e64.grad)
    p64.close()
    pmx.close()
