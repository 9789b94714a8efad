"""Batched evaluations (tlr_loglik_grad_batch through PlanBatch) and the inference drivers on the
device likelihood: the MLE with the device gradient, the observed information, and lockstep MCMC
chains whose every iteration is one batched call."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


def _data(case):
    d = np.load(os.path.join(GOLD, case + "_data.npz"))
    return d["S"], d["y"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_evaluations(tlr, precision):
    """Each plan of a batch computes exactly what it computes alone (same kernels, same inputs);
    a parameter vector whose factorization fails reports its failing tile without disturbing the
    others."""
    S, y = _data("n4000_b250")
    thetas = np.array([[1.0, 0.3, 0.05], [1.4, 0.25, 0.08], [0.7, 0.4, 0.03], [1.0, 0.3, 0.05]])
    pb = tlr.PlanBatch(4000, 250, 4, precision=precision)
    pb.set_data(S, y)
    out = pb.evaluate(thetas, "adaptive", 0.9)
    single = tlr.Plan(4000, 250)
    single.set_precision(precision)
    single.set_data(S, y)
    for q in range(4):
        ev = single.evaluate(thetas[q], "adaptive", 0.9, grad=True)
        ll, g, st = out[q]
        assert st == ev.status == 0
        assert ll == ev.loglik and np.array_equal(g, ev.grad)
    # fixed eps = 1e-3 fails at diagonal tile 3 on this field (reference golden value)
    out = pb.evaluate(thetas[:2], "fixed", 1e-3)
    ev = single.evaluate(thetas[0], "fixed", 1e-3, grad=True)
    assert out[0][2] == ev.status == 4 and out[0][0] is None
    pb.close()
    single.close()


def test_mle_and_observed_information(tlr):
    """L-BFGS-B with the device gradient reaches a stationary point at least as good as its start.
    The observed information (central differences of the device gradient) is symmetric positive
    definite and, with a tight rule (fixed eps = 1e-8, where the TLR likelihood is the dense one to
    ~1e-10), within 1e-3 of central differences of the dense FP64 gradient.  (Second differences
    of the adaptive-rule log-likelihood itself, the reference's method, codes/15:21-31, see the
    rank changes between stencil points; the device gradient freezes the ranks.)"""
    from adaptive_tlr_pilots_b200 import inference as I
    from oracle import tlr_oracle as O
    S, y = _data("n1030_b100")
    obj = I.TLRObjective(S, y, 100, "adaptive", 0.9, precision="mixed")
    x0 = np.log([1.5, 0.18, 0.1])
    r = I.mle(obj, x0)
    ll0, _ = obj(x0)
    assert r["loglik"] >= ll0 and r["failures"] == 0
    assert np.linalg.norm(r["grad_log"]) <= 1e-3 * max(1.0, abs(r["loglik"]))
    obj.close()
    tight = I.TLRObjective(S, y, 100, "fixed", 1e-8, precision="fp64")
    x = np.array(r["x_hat"])
    info = I.observed_information(tight, x, h=1e-4)
    H = info["info_log"]
    assert np.allclose(H, H.T) and np.all(np.linalg.eigvalsh(H) > 0)
    Hd = np.zeros((3, 3))
    h = 1e-4
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        gp = O.dense_loglik_and_grad(S, y, np.exp(x + e))[1] * np.exp(x + e)
        gm = O.dense_loglik_and_grad(S, y, np.exp(x - e))[1] * np.exp(x - e)
        Hd[:, a] = -(gp - gm) / (2 * h)
    Hd = 0.5 * (Hd + Hd.T)
    assert np.linalg.norm(H - Hd) <= 1e-3 * np.linalg.norm(Hd), (H, Hd)
    assert np.all(info["se_theta"] > 0)
    tight.close()


@pytest.mark.parametrize("kind", ["rw", "mala"])
def test_chains_run_in_batched_lockstep(tlr, kind):
    """Four chains from the reference's dispersed starts (multipliers of codes/35 and README), each
    iteration one batched call of four evaluations; chains stay in the prior box, accept at a
    reasonable rate and record no failed factorization."""
    from adaptive_tlr_pilots_b200 import inference as I
    S, y = _data("n1030_b100")
    obj = I.TLRObjective(S, y, 100, "adaptive", 0.9, precision="mixed", batch=4)
    theta = np.array([1.0, 0.3, 0.05])
    starts = np.log(theta * np.array([[1.3, 0.8, 1.5], [0.6, 1.4, 0.5], [2.0, 0.5, 2.0], [0.8, 1.2, 0.8]]))
    out = I.run_chains(obj, starts, iters=60, burn=50, seeds=[101, 102, 103, 104], kind=kind)
    ch = out["chain"]
    assert np.all(ch > I.LO) and np.all(ch < I.HI)
    assert all(f == 0 for f in out["failures"])
    assert 0.0 < np.mean(out["acceptance"]) < 1.0
    assert obj.evals >= 4 * 60
    obj.close()
