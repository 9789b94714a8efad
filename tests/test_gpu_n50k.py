"""Ranks at the headline size, N = 50,000, b = 500, adaptive tau = 0.9, theta = (1, 0.3, 0.05).

The reference's own tlr_cholesky run at this size (tests/golden/make_golden_n50k.py, about 7 minutes
on 8 cores) gives every initial (Sigma-tile) rank and every factor rank; they depend only on the
sites and theta, so the sites are drawn again here from the seed and the observations are zeros.
Bar: all 4,950 initial and 4,950 factor ranks identical, identical stored values, completed."""
import json
import os

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_n50k_ranks_match_reference():
    import adaptive_tlr_pilots_b200 as tlr
    g = json.load(open(os.path.join(GOLD, "golden_n50k.json")))
    S = O.simulate_sites(g["n"], seed=g["seed"])
    plan = tlr.Plan(g["n"], g["b"], cap=64, device=0)
    try:
        plan.set_precision("fp64")
        ev = plan.evaluate(g["theta"], g["rule"], g["value"], host_S=S, host_y=np.zeros(g["n"]))
    finally:
        plan.close()
        tlr.release_plans()
    sr, sw = np.asarray(ev.sigma_ranks), np.asarray(g["sigma_ranks"])
    assert np.array_equal(sr, sw), [(int(t), int(sr[t]), int(sw[t])) for t in np.flatnonzero(sr != sw)][:20]
    assert ev.info["stored_sigma"] == g["stored_sigma"]
    assert ev.info["completed"] == g["completed"]
    fr, fw = np.asarray(ev.factor_ranks), np.asarray(g["factor_ranks"])
    assert np.array_equal(fr, fw), [(int(t), int(fr[t]), int(fw[t])) for t in np.flatnonzero(fr != fw)][:20]
    assert ev.info["stored_factor"] == g["stored_factor"]
    assert ev.info["max_rank_factor"] == g["max_rank_factor"]
