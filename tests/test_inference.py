"""Inference drivers (MLE, observed information, lockstep MCMC, diagnostics) on analytic
densities: CPU-only checks of the host logic that drives the device likelihood."""
import numpy as np
import pytest

from adaptive_tlr_pilots_b200 import inference as I

MU = np.log([1.0, 0.3, 0.05])
PREC = np.array([[40.0, 5.0, 0.0], [5.0, 25.0, 3.0], [0.0, 3.0, 30.0]])


class Gauss:
    """log N(x; MU, PREC^{-1}) with its gradient; -inf (a 'failed factorization') where x[2] > fail."""

    def __init__(self, fail=np.inf):
        self.fail = fail
        self.calls = 0

    def __call__(self, x, grad=True):
        self.calls += 1
        x = np.asarray(x, dtype=np.float64)
        if x[2] > self.fail:
            return -np.inf, None
        d = x - MU
        return -0.5 * float(d @ PREC @ d), (-(PREC @ d) if grad else None)


def test_mle_reaches_the_mode():
    r = I.mle(Gauss(), MU + np.log([1.5, 0.6, 2.0]))
    np.testing.assert_allclose(r["x_hat"], MU, atol=1e-5)
    assert r["failures"] == 0 and r["success"]


def test_mle_counts_failures_and_still_converges():
    # the start is feasible; the first line search steps into the failing region and backtracks
    r = I.mle(Gauss(fail=MU[2] + 0.05), MU + np.array([1.5, -1.5, 0.04]))
    np.testing.assert_allclose(r["x_hat"], MU, atol=1e-4)
    assert r["failures"] >= 1


def test_observed_information_is_the_precision():
    r = I.observed_information(Gauss(), MU + 0.01)
    np.testing.assert_allclose(r["info_log"], PREC, rtol=1e-7, atol=1e-6)
    np.testing.assert_allclose(r["se_theta"], np.exp(MU + 0.01) * np.sqrt(np.diag(np.linalg.inv(PREC))), rtol=1e-6)


@pytest.mark.parametrize("kind", ["rw", "mala"])
def test_chains_sample_the_target(kind):
    obj = Gauss()
    starts = MU + np.array([[0.3, -0.3, 0.5], [-0.4, 0.4, -0.5], [0.6, -0.2, 0.3], [-0.2, 0.3, 0.0]])
    out = I.run_chains(obj, starts, iters=3000, burn=1000, seeds=[101, 102, 103, 104], kind=kind)
    post = out["chain"][:, 1000:].reshape(-1, 3)
    cov = np.linalg.inv(PREC)
    assert np.all(np.abs(post.mean(0) - MU) < 6 * np.sqrt(np.diag(cov) / 400)), (post.mean(0), MU)
    np.testing.assert_allclose(post.var(0), np.diag(cov), rtol=0.35)
    acc = np.array(out["acceptance"])
    assert np.all(acc > (0.15 if kind == "rw" else 0.35)) and np.all(acc < (0.5 if kind == "rw" else 0.85))
    for j in range(3):
        rh, ess = I.split_rhat_ess(out["chain"][:, 1000:, j])
        assert rh < 1.05 and ess > 100


def test_failed_evaluations_are_rejected_and_counted():
    obj = Gauss(fail=MU[2] + 0.05)
    out = I.run_chains(obj, MU[None, :], iters=400, burn=200, seeds=[7], kind="rw")
    assert out["failures"][0] > 0
    assert np.all(out["chain"][0, :, 2] <= MU[2] + 0.05)


@pytest.mark.parametrize("kind", ["rw", "mala"])
def test_resume_from_checkpoint_is_identical(tmp_path, kind):
    starts = MU + np.array([[0.2, 0.1, -0.1], [-0.1, 0.2, 0.1]])
    full = I.run_chains(Gauss(), starts, iters=300, burn=150, seeds=[1, 2], kind=kind)
    ck = str(tmp_path / "ck.npz")
    part = I.run_chains(Gauss(), starts, iters=200, burn=150, seeds=[1, 2], kind=kind, ckpt=ck, ckpt_every=100)
    np.testing.assert_array_equal(part["chain"], full["chain"][:, :200])
    # a longer run picks the state up at iteration 200 and continues
    res = I.run_chains(Gauss(), starts, iters=300, burn=150, seeds=[1, 2], kind=kind, ckpt=ck, ckpt_every=100)
    np.testing.assert_array_equal(res["chain"], full["chain"])
    np.testing.assert_array_equal(res["lls"], full["lls"])


def test_split_rhat_flags_chains_that_disagree():
    rng = np.random.default_rng(0)
    good = rng.standard_normal((4, 2000))
    rh, ess = I.split_rhat_ess(good)
    assert abs(rh - 1.0) < 0.01 and ess > 4000
    bad = good + np.array([0.0, 0.0, 1.0, 1.0])[:, None]
    assert I.split_rhat_ess(bad)[0] > 1.1


def _direct_split_rhat_ess(chains):
    """Direct-sum restatement of the same estimator (scipy ranks, lag-by-lag autocovariances,
    an explicit loop for Geyer's initial monotone sequence) to check the vectorised one."""
    from scipy import stats
    x = np.asarray(chains, float)
    h = x.shape[1] // 2
    seq = np.vstack([x[:, :h], x[:, h:2 * h]])
    r = stats.rankdata(seq, method="average").reshape(seq.shape)
    z = stats.norm.ppf((r - 0.375) / (seq.size + 0.25))
    m = z.shape[0]
    W = np.mean([np.var(c, ddof=1) for c in z])
    vp = (h - 1) / h * W + np.var(z.mean(1), ddof=1)
    rho = []
    for t in range(h):
        ac = np.mean([np.dot(c[:h - t] - c.mean(), c[t:] - c.mean()) / h for c in z])
        rho.append(1.0 - (W - ac) / vp)
    tau, prev = -1.0, np.inf
    for t in range(0, h - 1, 2):
        p = rho[t] + rho[t + 1]
        if p < 0:
            break
        prev = min(prev, p)
        tau += 2.0 * prev
    tau = max(tau, 1.0 / np.log10(m * h))
    return np.sqrt(vp / W), m * h / tau


def test_split_rhat_ess_matches_direct_sums_and_ar1_theory():
    rng = np.random.default_rng(3)
    phi, M, n = 0.8, 4, 4000
    x = np.zeros((M, n))
    e = rng.standard_normal((M, n)) * np.sqrt(1 - phi * phi)
    x[:, 0] = rng.standard_normal(M)
    for t in range(1, n):
        x[:, t] = phi * x[:, t - 1] + e[:, t]
    x[1, 100:110] = x[1, 99]  # tied draws take their average rank
    rh, ess = I.split_rhat_ess(x)
    rh_d, ess_d = _direct_split_rhat_ess(x)
    assert abs(rh - rh_d) < 1e-12 and abs(ess - ess_d) < 1e-8 * ess_d
    # AR(1): integrated autocorrelation time (1 + phi) / (1 - phi) = 9
    assert 0.75 < ess / (M * n / 9.0) < 1.3


def test_autotune_table_lookup(tmp_path):
    """best_workspaces takes the fastest measured count for the nearest tuned N with the same tile
    size, rule and precision, capped at the batch; the default without a matching entry."""
    import json as _json

    from adaptive_tlr_pilots_b200 import autotune as A
    path = str(tmp_path / "t.json")
    assert A.best_workspaces(50000, 500, 64, path=path) == A.DEFAULT_WORKSPACES
    table = {"a": dict(n=50000, b=500, rule="adaptive", value=0.9, precision="mixed", best=6,
                       evals_per_s={"4": 5.0, "6": 6.0}),
             "b": dict(n=20000, b=500, rule="adaptive", value=0.9, precision="mixed", best=2,
                       evals_per_s={"2": 9.0}),
             "c": dict(n=50000, b=250, rule="adaptive", value=0.9, precision="mixed", best=8,
                       evals_per_s={"8": 1.0})}
    _json.dump(table, open(path, "w"))
    assert A.best_workspaces(60000, 500, 64, path=path) == 6
    assert A.best_workspaces(18000, 500, 64, path=path) == 2
    assert A.best_workspaces(50000, 500, 3, path=path) == 3
    assert A.best_workspaces(50000, 500, 64, precision="fp64", path=path) == A.DEFAULT_WORKSPACES
