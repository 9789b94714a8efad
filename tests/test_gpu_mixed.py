"""The mixed-precision path (three-pass sketches bounded by the exact FP64 residual, split-TF32
tensor-core GEMMs in the backward pass) against the FP64 parity path and the dense FP64 likelihood.

Budget (the accuracy contract of the mixed path): |loglik_mixed - loglik_fp64| <= 1e-2 nats and a
gradient within 1e-3 (relative, 2-norm) of the FP64 path's on the same inputs and rule; PD
verdicts identical.  With a tight rule the mixed log-likelihood and gradient are also checked
against the dense FP64 oracle."""
import os

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

CASES = [
    ("n1030_b100", 100, (1.0, 0.3, 0.05)),
    ("n4000_b250", 250, (1.0, 0.3, 0.05)),
    ("n2000_b200_r1.0_e0.005", 200, (1.0, 1.0, 0.005)),
    ("n1500_b250_s2.5_r0.1", 250, (2.5, 0.1, 0.05)),
]


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


def _eval(tlr, d, b, theta, rule, value, precision):
    n = len(d["y"])
    p = tlr.Plan(n, b)
    p.set_precision(precision)
    p.set_data(d["S"], d["y"])
    ev = p.evaluate(theta, rule, value, grad=True)
    ev2 = p.evaluate(theta, rule, value, grad=True)
    p.close()
    return ev, ev2


@pytest.mark.parametrize("case,b,theta", CASES)
@pytest.mark.parametrize("rule,value", [("adaptive", 0.9), ("fixed", 1e-4)])
def test_mixed_within_budget_of_fp64(tlr, case, b, theta, rule, value):
    d = np.load(os.path.join(GOLD, case + "_data.npz"))
    e64, _ = _eval(tlr, d, b, theta, rule, value, "fp64")
    emx, emx2 = _eval(tlr, d, b, theta, rule, value, "mixed")
    assert emx.status == e64.status  # same PD verdict (and failing tile)
    if e64.status != 0:
        assert emx.info["failed_at"] == e64.info["failed_at"]
        return
    assert abs(emx.loglik - e64.loglik) <= 1e-2
    assert np.linalg.norm(emx.grad - e64.grad) <= 1e-3 * np.linalg.norm(e64.grad), (emx.grad, e64.grad)
    # the initial compression ranks are the FP64 ones up to ties (three-pass sketch, exact residual)
    assert np.mean(emx.sigma_ranks != e64.sigma_ranks) <= 0.02
    # bit-identical on a repeat (fixed reduction orders everywhere)
    assert emx2.loglik == emx.loglik and np.array_equal(emx2.grad, emx.grad)


def test_mixed_close_to_dense_for_tight_rule(tlr):
    """fixed eps = 1e-8: the mixed log-likelihood within 1e-6 relative and the gradient within 1e-4
    (relative) of the dense FP64 oracle."""
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    theta = (1.0, 0.3, 0.05)
    emx, _ = _eval(tlr, d, 100, theta, "fixed", 1e-8, "mixed")
    ll_d, g_d = O.dense_loglik_and_grad(d["S"], d["y"], np.array(theta))
    assert abs(emx.loglik - ll_d) <= 1e-6 * abs(ll_d)
    assert np.linalg.norm(emx.grad - g_d) <= 1e-4 * np.linalg.norm(g_d)
