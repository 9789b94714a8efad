"""The CPU oracle against the reference's own outputs (tests/golden, made by make_golden.py)
and against the values the reference committed for N = 10,000."""
import json
import os

import numpy as np
import pytest

from oracle import tlr_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load_gold():
    return json.load(open(os.path.join(GOLD, "golden.json")))


def test_tile_bounds():
    assert O.tile_bounds(10, 4) == [(0, 4), (4, 8), (8, 10)]
    assert O.tile_bounds(8, 4) == [(0, 4), (4, 8)]
    assert O.tile_bounds(3, 5) == [(0, 3)]


def test_morton_matches_reference():
    d = np.load(os.path.join(GOLD, "morton_case.npz"))
    np.testing.assert_array_equal(O.morton_order(d["xy"]), d["perm"])


@pytest.mark.parametrize("case", [c["name"] for c in load_gold()["cases"]])
def test_oracle_matches_reference(case):
    gold = {c["name"]: c for c in load_gold()["cases"]}[case]
    d = np.load(os.path.join(GOLD, gold["data"]))
    S, y = d["S"], d["y"]
    bounds = O.tile_bounds(gold["n"], gold["b"])
    ll_dense, _ = O.loglik_dense(O.cov_dense(S, gold["theta"]), y)
    assert abs(ll_dense - gold["dense_loglik"]) <= 1e-10 * abs(gold["dense_loglik"])
    for rec in gold["rules"]:
        ll, fac, info = O.tlr_loglik(S, y, gold["theta"], bounds, rec["rule"], rec["value"])
        assert info["sigma_ranks"] == rec["sigma_ranks"]
        assert info["stored_sigma"] == rec["stored_sigma"]
        assert info["completed"] == rec["completed"]
        if rec["completed"]:
            assert info["factor_ranks"] == rec["factor_ranks"]
            assert info["stored_factor"] == rec["stored_factor"]
            assert abs(ll - rec["loglik"]) <= 1e-10 * abs(rec["loglik"])
        else:
            assert info["failed_at"] == rec["failed_at"]


@pytest.mark.slow
def test_oracle_reproduces_committed_n10000():
    """results/tlr_cholesky/tlr_cholesky_n10000.json: dense and TLR log-likelihoods on the
    reference's own simulated field (regenerated here by the same seeded protocol)."""
    com = load_gold()["committed_n10000"]
    S, y, _, _ = O.simulate_field(10000)
    bounds = O.tile_bounds(10000, 250)
    ll_dense, _ = O.loglik_dense(O.cov_dense(S, (1.0, 0.3, 0.05)), y)
    assert abs(ll_dense - com["dense_loglik"]) <= 1e-9 * abs(com["dense_loglik"])
    for rec in com["rules"]:
        if rec["rule"] != "adaptive" and rec["value"] not in (1e-3, 1e-4):
            continue
        ll, _, info = O.tlr_loglik(S, y, (1.0, 0.3, 0.05), bounds, rec["rule"], rec["value"])
        assert info["stored_sigma"] == rec["stored_sigma"]
        assert info["completed"] == rec["completed"]
        if rec["completed"]:
            assert info["stored_factor"] == rec["stored_factor"]
            assert info["max_rank_factor"] == rec["max_rank_factor"]
            assert abs(info["mean_rank_factor"] - rec["mean_rank_factor"]) < 1e-12
            assert abs((ll - ll_dense) - rec["loglik_err"]) <= 1e-7
        else:
            assert info["failed_at"] == rec["failed_at_tile"]


def test_frozen_ranks_replay():
    """Replaying the recorded ranks at the same theta gives the same log-likelihood."""
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    S, y = d["S"], d["y"]
    bounds = O.tile_bounds(1030, 100)
    log = {}
    ll, _, _ = O.tlr_loglik(S, y, (1.0, 0.3, 0.05), bounds, "adaptive", 0.9, rank_log=log)
    ll2, _, _ = O.tlr_loglik(S, y, (1.0, 0.3, 0.05), bounds, "adaptive", 0.9, frozen=log)
    assert ll == ll2


def test_dense_gradient_matches_finite_differences():
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    S, y = d["S"][:300], d["y"][:300]
    th = np.array([1.0, 0.3, 0.05])
    _, g = O.dense_loglik_and_grad(S, y, th)
    for a in range(3):
        h = 1e-5 * th[a]
        tp, tm = th.copy(), th.copy()
        tp[a] += h; tm[a] -= h
        fd = (O.loglik_dense(O.cov_dense(S, tp), y)[0] - O.loglik_dense(O.cov_dense(S, tm), y)[0]) / (2 * h)
        assert abs(fd - g[a]) <= 1e-5 * max(1.0, abs(g[a]))


def test_oracle_prediction_matches_reference():
    """The restated kriging, factor product, solves and skill scores reproduce the reference's own
    outputs on the N = 1,030 field (fixture from tests/golden/make_golden_predict.py)."""
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    f = np.load(os.path.join(GOLD, "predict_n1030.npz"))
    S, y = d["S"], d["y"]
    theta = (1.0, 0.3, 0.05)
    bounds = O.tile_bounds(len(y), 100)
    ll, fac, _ = O.tlr_loglik(S, y, theta, bounds, "adaptive", 0.9)
    assert abs(ll - float(f["loglik"])) <= 1e-10 * abs(ll)
    mu, sd = O.tlr_predict(S, y, f["Sp"], theta, bounds, fac)
    np.testing.assert_allclose(mu, f["mu"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(sd, f["sd"], rtol=1e-9)
    np.testing.assert_allclose(O.tlr_matvec_L(fac[0], fac[1], bounds, f["z"][:, None])[:, 0], f["Lz"], rtol=1e-9,
                               atol=1e-12)
    fwd = O.tlr_forward(fac[0], fac[1], bounds, y[:, None])[:, 0]
    np.testing.assert_allclose(fwd, f["fwd"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(O.tlr_backward(fac[0], fac[1], bounds, fwd[:, None])[:, 0], f["bwd"], rtol=1e-9,
                               atol=1e-12)
    sk = O.skill(f["yp"], f["mu"], f["sd"])
    assert abs(sk["rmse"] - float(f["rmse"])) <= 1e-12 and abs(sk["crps"] - float(f["crps"])) <= 1e-12
    assert sk["cover90"] == float(f["cover90"])


@pytest.mark.parametrize("case", ["n1030_b100", "n4000_b250"])
def test_oracle_matern52_matches_reference(case):
    """With nu = 2.5 (the kernel codes/24_screening_stress.py patches into 17) the oracle gives the
    reference's ranks, stored values, TLR and dense log-likelihoods (golden_nu52.json)."""
    gold = {c["name"]: c for c in json.load(open(os.path.join(GOLD, "golden_nu52.json")))["cases"]}[case]
    d = np.load(os.path.join(GOLD, gold["data"]))
    S, y = d["S"], d["y"]
    bounds = O.tile_bounds(gold["n"], gold["b"])
    O.set_kernel(2.5)
    try:
        for rec in gold["rules"]:
            ll, _, info = O.tlr_loglik(S, y, gold["theta"], bounds, rec["rule"], rec["value"])
            assert info["sigma_ranks"] == rec["sigma_ranks"]
            assert info["completed"] == rec["completed"]
            assert info["factor_ranks"] == rec["factor_ranks"]
            assert info["stored_factor"] == rec["stored_factor"]
            assert abs(ll - rec["loglik"]) <= 1e-10 * abs(rec["loglik"])
        ll_d, _ = O.loglik_dense(O.cov_dense(S, gold["theta"]), y)
        assert abs(ll_d - gold["dense_loglik"]) <= 1e-10 * abs(gold["dense_loglik"])
    finally:
        O.set_kernel(1.5)


def test_oracle_assembled_rule_matches_reference():
    """The oracle's truncate_tiles + loglik_dense against the reference's own outputs
    (codes/11_tlr_rank_rules.py:74-126 run by tests/golden/make_golden_assembled.py)."""
    g = json.load(open(os.path.join(GOLD, "golden_assembled.json")))
    d = np.load(os.path.join(GOLD, g["data"]))
    S, y = d["S"], d["y"]
    theta = tuple(g["theta"])
    bounds = O.tile_bounds(g["n"], g["b"])
    for rec in g["rules"]:
        K = O.cov_dense(S, theta)
        stored, max_rel, max_abs, fro, ranks = O.truncate_tiles(K, bounds, rec["rule"], rec["value"],
                                                                theta[0] * theta[2])
        assert stored == rec["stored"] and ranks == rec["ranks"]
        np.testing.assert_allclose([max_rel, max_abs, fro], [rec["max_rel"], rec["max_abs"], rec["fro_err"]],
                                   rtol=1e-9)
        ll = O.loglik_dense(K, y)[0]
        if rec["loglik"] is None:
            assert ll is None
        else:
            assert abs(ll - rec["loglik"]) <= 1e-10 * abs(rec["loglik"])


@pytest.mark.parametrize("q", [0, 1, 2])
def test_oracle_mixed_storage_rule_matches_reference(q):
    """Rule 'mixed' (codes/17_tlr_cholesky_pilot.py:33-82): the oracle against the reference's
    own outputs (tests/golden/make_golden_mixed_rule.py): ranks and storage precision of every
    factor tile, stored bytes, log-likelihood."""
    rec = json.load(open(os.path.join(GOLD, "golden_mixed_rule.json")))["cases"][q]
    d = np.load(os.path.join(GOLD, rec["data"]))
    bounds = O.tile_bounds(rec["n"], rec["b"])
    ll, _, info = O.tlr_loglik(d["S"], d["y"], tuple(rec["theta"]), bounds, "mixed", rec["tau"])
    assert info["factor_ranks"] == rec["factor_ranks"]
    assert info["factor_prec"] == rec["factor_prec"]
    assert info["stored_factor_bytes"] == rec["stored_factor_bytes"]
    assert {str(k): v for k, v in info["precision_mix_factor_tiles"].items()} == rec["precision_mix_factor_tiles"]
    assert abs(ll - rec["loglik"]) <= 1e-10 * abs(rec["loglik"])
