"""The assembled-matrix rule on the device against the reference's outputs.

codes/11_tlr_rank_rules.py:74-126 (truncate_tiles inside make_cov, then loglik_dense) and
codes/19_tlr_mcmc_gpu.py:27-138 (Likelihood: the same Sigma^TLR through a dense Cholesky), run by
tests/golden/make_golden_assembled.py on the N = 4,000, b = 250 field.  Bar: identical tile ranks
and stored values, the reference's error statistics (max relative / absolute tile error,
||Sigma - Sigma^TLR||_F) to 1e-6 relative, the log-likelihood of Sigma^TLR to 1e-10 relative and
the same positive-definiteness verdict.  The reference's svd_mode 'fp32' and 'rand' may keep more
directions than the minimal rank; here every mode gives the minimal ('fp64') ranks, so for those
modes the check is stored <= the reference's and the log-likelihood within 1e-3 nats."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def case():
    import adaptive_tlr_pilots_b200 as tlr
    g = json.load(open(os.path.join(GOLD, "golden_assembled.json")))
    d = np.load(os.path.join(GOLD, g["data"]))
    yield tlr, g, d["S"], d["y"]
    tlr.release_plans()


def test_make_cov_and_loglik_match_reference(case):
    tlr, g, S, y = case
    bounds = tlr.tile_bounds(g["n"], g["b"])
    for rec in g["rules"]:
        K, info = tlr.make_cov(S, g["theta"], rec["rule"], rec["value"], bounds)
        stored, max_rel, max_abs, fro, ranks = info
        assert stored == rec["stored"] and ranks == rec["ranks"], rec["rule"]
        np.testing.assert_allclose([max_rel, max_abs, fro], [rec["max_rel"], rec["max_abs"], rec["fro_err"]],
                                   rtol=1e-6)
        # symmetric, exact diagonal tiles
        assert float((K - K.T).abs().max()) == 0.0
        ll, _ = tlr.loglik_dense_K(K, y)
        if rec["loglik"] is None:
            assert ll is None
        else:
            assert abs(ll - rec["loglik"]) <= 1e-10 * abs(rec["loglik"]), (ll, rec["loglik"])


def test_assembled_tiles_match_oracle_truncations(case):
    """Every entry of Sigma^TLR against the oracle's truncate_tiles (exact SVD truncations)."""
    from oracle import tlr_oracle as O
    tlr, g, S, y = case
    bounds = tlr.tile_bounds(g["n"], g["b"])
    K, _ = tlr.make_cov(S, g["theta"], "adaptive", 0.9, bounds)
    Ko = O.cov_dense(S, tuple(g["theta"]))
    O.truncate_tiles(Ko, bounds, "adaptive", 0.9, g["theta"][0] * g["theta"][2])
    assert np.abs(K.cpu().numpy() - Ko).max() <= 1e-11


@pytest.mark.parametrize("mode", ["fp64", "fp32", "rand"])
def test_likelihood_19_matches_reference(case, mode):
    tlr, g, S, y = case
    L = tlr.Likelihood(S, y, g["b"], 0, svd_mode=mode)
    for rec in g["rules"]:
        ref = rec["likelihood19"][mode]
        v = L(g["theta"], rec["rule"], rec["value"])
        assert L.last["ok"] == ref["ok"]
        if not ref["ok"]:
            assert v == -float("inf")
            continue
        if mode == "fp64":
            assert L.last["stored"] == ref["stored"]
            assert abs(v - ref["loglik"]) <= 1e-10 * abs(ref["loglik"]), (v, ref["loglik"])
        else:
            assert L.last["stored"] <= ref["stored"]
            assert abs(v - ref["loglik"]) <= 1e-3
    dense = L(g["theta"], "dense", None)
    assert abs(dense - tlr.dense_loglik(S, y, g["theta"])) <= 1e-10 * abs(dense)
