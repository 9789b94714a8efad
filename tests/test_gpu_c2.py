"""Parity at N = 20,000, b = 500: the range x nugget sweep, range in {0.1, 0.3, 1.0} x eta in
{0.05, 0.005}, adaptive tau = 0.9, every field simulated with its own theta.

The fixtures come from running the reference's own tlr_loglik (codes/17_tlr_cholesky_pilot.py:
259-266) and truncate_svd (17:107-116) on these fields (tests/golden/make_golden_c2.py).  Bar, as
for the small cases: identical initial and factor ranks (780 tiles each), identical PD verdict,
stored values, relative log-likelihood error <= 1e-10.  The mixed-precision path is held to its
budget on the same fields: |loglik_mixed - loglik_fp64| <= 1e-2 nats, same PD verdict."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
REL_TOL = 1e-10


def _gold():
    return json.load(open(os.path.join(GOLD, "golden_c2.json")))


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


@pytest.fixture(scope="module")
def fields():
    g = _gold()
    d = np.load(os.path.join(GOLD, g["data"]))
    return g, d["S"], {c["name"]: d["y_" + c["name"]] for c in g["cases"]}


@pytest.mark.parametrize("name", [c["name"] for c in _gold()["cases"]])
def test_sweep_matches_reference(tlr, fields, name):
    g, S, ys = fields
    rec = {c["name"]: c for c in g["cases"]}[name]
    plan = tlr.get_plan(g["n"], g["b"])
    plan.set_precision("fp64")
    ev = plan.evaluate(rec["theta"], g["rule"], g["value"], host_S=S, host_y=ys[name])
    sr = np.asarray(ev.sigma_ranks)
    want = np.asarray(rec["sigma_ranks"])
    assert np.array_equal(sr, want), [(int(t), int(sr[t]), int(want[t])) for t in np.flatnonzero(sr != want)]
    assert ev.info["stored_sigma"] == rec["stored_sigma"]
    assert ev.info["completed"] == rec["completed"]
    if not rec["completed"]:
        assert ev.info["failed_at"] == rec["failed_at"]
        return
    fr = np.asarray(ev.factor_ranks)
    fw = np.asarray(rec["factor_ranks"])
    assert np.array_equal(fr, fw), [(rec["factor_keys"][t], int(fr[t]), int(fw[t])) for t in np.flatnonzero(fr != fw)]
    assert ev.info["stored_factor"] == rec["stored_factor"]
    assert ev.info["max_rank_factor"] == rec["max_rank_factor"]
    rel = abs(ev.loglik - rec["loglik"]) / abs(rec["loglik"])
    assert rel <= REL_TOL, (ev.loglik, rec["loglik"], rel)
    assert abs(ev.info["logdet"] - rec["logdet"]) <= 10 * REL_TOL * abs(rec["logdet"])


@pytest.mark.parametrize("name", [c["name"] for c in _gold()["cases"]])
def test_sweep_mixed_within_budget(tlr, fields, name):
    g, S, ys = fields
    rec = {c["name"]: c for c in g["cases"]}[name]
    plan = tlr.get_plan(g["n"], g["b"])
    plan.set_precision("mixed")
    try:
        ev = plan.evaluate(rec["theta"], g["rule"], g["value"], host_S=S, host_y=ys[name])
    finally:
        plan.set_precision("fp64")
    assert ev.info["completed"] == rec["completed"]
    if rec["completed"]:
        assert abs(ev.loglik - rec["loglik"]) <= 1e-2, (ev.loglik, rec["loglik"])
