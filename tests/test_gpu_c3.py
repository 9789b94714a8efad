"""The differentiated likelihood at N = 20,000, b = 500 (16 parameter vectors).

theta is drawn log-uniform within a factor of 3 of (1, 0.3, 0.05) (seed 20261021) on the
N = 20,000 field simulated at (1, 0.3, 0.05) by the reference's protocol (the fixture of
tests/golden/make_golden_c2.py).  At every theta the device gradient (ranks frozen, selected
inversion) is compared with

  * central differences of the frozen-rank TLR log-likelihood (step 1e-5 relative, FP64), the
    ranks recorded at theta and replayed at theta +- h through the plan's rank map, and
  * the dense FP64 gradient 1/2 a^T dS a - 1/2 tr(S^-1 dS) (Cholesky on the device).

The reference has no gradient (its only derivative is the finite-difference Hessian of
codes/15_pilot_standard_errors.py:21-31); these are the checks the gradient is held to.  With the
adaptive rule (tau = 0.9) the TLR gradient differs from both by the truncation; measured on a B200:
at most 1.03e-3 from the frozen-rank differences and 2.6e-4 from the dense gradient over the 16
points (so within the 1e-3 relative gradient budget against dense FP64), and the bounds below are
those with a margin.  With a tight rule (fixed eps = 1e-8) all three agree to 1.7e-5 (bound 1e-4)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
THETA0 = np.array([1.0, 0.3, 0.05])
FD_REL = 1e-5
TOL_FD_ADAPTIVE = 2e-3      # |g - fd| / |fd|, adaptive tau = 0.9
TOL_DENSE_ADAPTIVE = 1e-3   # |g - g_dense| / |g_dense|, adaptive tau = 0.9
TOL_TIGHT = 1e-4            # both, fixed eps = 1e-8


def thetas16():
    rng = np.random.default_rng(20261021)
    return THETA0[None, :] * np.exp(rng.uniform(-np.log(3.0), np.log(3.0), (16, 3)))


@pytest.fixture(scope="module")
def setup():
    import adaptive_tlr_pilots_b200 as tlr
    from adaptive_tlr_pilots_b200 import synth
    g = json.load(open(os.path.join(GOLD, "golden_c2.json")))
    d = np.load(os.path.join(GOLD, g["data"]))
    S, y = d["S"], d["y_r0.3_e0.05"]
    plan = tlr.Plan(g["n"], g["b"], cap=64, device=0)
    plan.set_data(S, y)
    plan.set_precision("fp64")
    yield tlr, synth, plan, S, y
    plan.close()
    tlr.release_plans()


def _grad_fd(plan, theta, rule, value):
    plan.rank_map("record")
    ev = plan.evaluate(theta, rule, value, grad=True)
    assert ev.status == 0, ev.info
    plan.rank_map("replay")
    fd = np.zeros(3)
    try:
        for a in range(3):
            h = FD_REL * theta[a]
            tp, tm = theta.copy(), theta.copy()
            tp[a] += h
            tm[a] -= h
            lp = plan.evaluate(tp, rule, value).loglik
            lm = plan.evaluate(tm, rule, value).loglik
            fd[a] = (lp - lm) / (2.0 * h)
    finally:
        plan.rank_map("rule")
    return ev.loglik, np.asarray(ev.grad), fd


def test_sixteen_thetas_adaptive(setup):
    tlr, synth, plan, S, y = setup
    rows = []
    for theta in thetas16():
        ll, g, fd = _grad_fd(plan, theta, "adaptive", 0.9)
        lld, gd = synth.dense_loglik_grad_gpu(S, y, tuple(theta), device=0)
        gd = np.asarray(gd)
        rows.append((theta.tolist(), float(np.linalg.norm(g - fd) / np.linalg.norm(fd)),
                     float(np.linalg.norm(g - gd) / np.linalg.norm(gd)), abs(ll - lld)))
    print(json.dumps(rows))
    assert max(r[1] for r in rows) <= TOL_FD_ADAPTIVE, rows
    assert max(r[2] for r in rows) <= TOL_DENSE_ADAPTIVE, rows


@pytest.mark.parametrize("q", [0, 7])
def test_tight_rule_agrees_with_fd_and_dense(setup, q):
    tlr, synth, plan, S, y = setup
    theta = thetas16()[q]
    ll, g, fd = _grad_fd(plan, theta, "fixed", 1e-8)
    lld, gd = synth.dense_loglik_grad_gpu(S, y, tuple(theta), device=0)
    gd = np.asarray(gd)
    assert np.linalg.norm(g - fd) <= TOL_TIGHT * np.linalg.norm(fd), (g, fd)
    assert np.linalg.norm(g - gd) <= TOL_TIGHT * np.linalg.norm(gd), (g, gd)
    assert abs(ll - lld) <= 1e-6 * abs(lld)


def test_replayed_ranks_reproduce_the_recorded_evaluation(setup):
    """Replaying the map at the recording theta gives the recorded evaluation bit for bit."""
    tlr, synth, plan, S, y = setup
    theta = thetas16()[3]
    plan.rank_map("record")
    a = plan.evaluate(theta, "adaptive", 0.9)
    plan.rank_map("replay")
    try:
        b = plan.evaluate(theta, "adaptive", 0.9)
    finally:
        plan.rank_map("rule")
    assert a.loglik == b.loglik
    assert list(a.factor_ranks) == list(b.factor_ranks)
