"""The storage-precision rule 'mixed' on the device against the reference's outputs.

codes/17_tlr_cholesky_pilot.py rule 'mixed' (17:33-82, 145-148, 163-164, 183-184, 203-204,
210-214): adaptive ranks, every stored factor pair rounded to the fewest of FP8 / FP16 / FP32 /
FP64 bits whose rounding error fits the budget left after truncation, the factorization carried
on with the rounded factors (the recompressions then QR them in general form).  Fixtures from
running the reference (tests/golden/make_golden_mixed_rule.py).  Bar, as for the other rules:
identical factor ranks, identical storage precision of every factor tile, stored bytes and
precision mix, relative log-likelihood error <= 1e-10."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _cases():
    return json.load(open(os.path.join(GOLD, "golden_mixed_rule.json")))["cases"]


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


@pytest.mark.parametrize("q", range(len(_cases())))
def test_mixed_rule_matches_reference(tlr, q):
    rec = _cases()[q]
    d = np.load(os.path.join(GOLD, rec["data"]))
    plan = tlr.get_plan(rec["n"], rec["b"])
    plan.set_precision("fp64")
    ev = plan.evaluate(rec["theta"], "mixed", rec["tau"], host_S=d["S"], host_y=d["y"])
    assert ev.info["completed"] == rec["completed"]
    fr = np.asarray(ev.factor_ranks)
    assert list(fr) == rec["factor_ranks"]
    got, want = np.asarray(ev.info["factor_prec"]), np.asarray(rec["factor_prec"])
    assert np.array_equal(got, want), [(t, int(got[t]), int(want[t])) for t in np.flatnonzero(got != want)]
    assert ev.info["stored_factor_bytes"] == rec["stored_factor_bytes"]
    assert {str(k): v for k, v in ev.info["precision_mix_factor_tiles"].items()} == rec["precision_mix_factor_tiles"]
    assert abs(ev.loglik - rec["loglik"]) <= 1e-10 * abs(rec["loglik"]), (ev.loglik, rec["loglik"])
    # the drop-in call surface carries the reference's info keys
    bounds = tlr.tile_bounds(rec["n"], rec["b"])
    ll, fac, info = tlr.tlr_loglik(d["S"], d["y"], rec["theta"], bounds, "mixed", rec["tau"])
    assert info["factor_bytes_frac"] == pytest.approx(rec["factor_bytes_frac"], rel=1e-12)
    assert abs(ll - rec["loglik"]) <= 1e-10 * abs(rec["loglik"])
