"""The storage-precision rule 'mixed' on the device against the reference.

codes/17_tlr_cholesky_pilot.py rule 'mixed' (17:33-82, 145-148, 163-164, 183-184, 203-204,
210-214): adaptive ranks, every stored factor pair rounded to the fewest of FP8 / FP16 / FP32 /
FP64 bits whose rounding error fits the budget left after truncation, the factorization carried
on with the rounded factors (the recompressions then QR them in general form).  Fixtures from
running the reference (tests/golden/make_golden_mixed_rule.py); the oracle reproduces them
exactly (tests/test_oracle.py).

The rule is ill-conditioned in its inputs: FP16 storage turns a 1e-13 difference in one factor
entry into a 2^-11 jump when the entry lies near a rounding boundary, and many of its rank and
storage decisions sit within a few percent of their budgets.  The reference itself, run on its
sites times (1 + 1e-13 z), moves its log-likelihood by up to 0.42 nats on these fields and changes
ranks and storage bits (the fixture's `perturbed_1e-13` runs).  Even with every rank and storage
decision fixed, single entries that land within 1e-11 of an FP16 rounding boundary round to the
other neighbour in one implementation or the other and the difference spreads through the
factorization (measured on a B200 with the oracle's decisions replayed: 4.2e-3 and 9.4e-5 relative
on the two N = 4,000 fields, 2e-11 on the N = 1,030 field, where no entry is that close).  So:

  * the N = 1,030 field matches the reference exactly (ranks, storage bits, bytes, the
    log-likelihood to 1e-9 relative): the arithmetic of the rule, the device being bit-reproducible;
  * with every decision replayed (the oracle's ranks and storage bits loaded into the plan's rank
    map): identical ranks, storage bits and stored bytes on every field;
  * free running, every field: the log-likelihood within the reference's own spread under the
    1e-13 perturbations (widened by half its width), stored bytes within 1 %, every precision
    count within 5 tiles of the reference's."""
import json
import os

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
EXACT_REL_TOL = 1e-9


def _cases():
    return json.load(open(os.path.join(GOLD, "golden_mixed_rule.json")))["cases"]


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


def _device_map(log, nB, size):
    """The oracle's decision log in the plan's rank-map layout: initial tile t = i (i - 1) / 2 + j,
    then per step k its trailing pairs (i, j), k < j < i, at ii (ii - 1) / 2 + jj (ii = i - k - 1,
    jj = j - k - 1); the panel solves' storage bits after all of those."""
    ntiles = nB * (nB - 1) // 2
    ranks = np.zeros(size, dtype=np.int32)
    bits = np.full(size + ntiles, 64, dtype=np.int32)
    off = [ntiles]
    for k in range(nB):
        mB = nB - k - 1
        off.append(off[-1] + mB * (mB - 1) // 2)
    for key, v in log.items():
        if key[0] in ("init", "init_bits"):
            _, i, j = key
            pos = i * (i - 1) // 2 + j
        elif key[0] in ("rc", "rc_bits"):
            _, k, i, j = key
            ii, jj = i - k - 1, j - k - 1
            pos = off[k] + ii * (ii - 1) // 2 + jj
        else:  # trsm_bits (i, k)
            _, i, k = key
            bits[size + i * (i - 1) // 2 + k] = v
            continue
        if key[0].endswith("bits"):
            bits[pos] = v
        else:
            ranks[pos] = v
    return ranks, bits


@pytest.mark.parametrize("q", range(len(_cases())))
def test_mixed_rule_with_replayed_decisions(tlr, q):
    rec = _cases()[q]
    d = np.load(os.path.join(GOLD, rec["data"]))
    bounds = O.tile_bounds(rec["n"], rec["b"])
    log = {}
    ll_o, _, info_o = O.tlr_loglik(d["S"], d["y"], tuple(rec["theta"]), bounds, "mixed", rec["tau"], rank_log=log)
    plan = tlr.Plan(rec["n"], rec["b"], cap=64, device=0)
    try:
        plan.set_data(d["S"], d["y"])
        ranks, bits = _device_map(log, plan.nB, int(plan.lib.tlr_plan_rank_map_size(plan.handle)))
        plan.rank_map_set(ranks, bits)
        plan.rank_map("replay")
        ev = plan.evaluate(rec["theta"], "mixed", rec["tau"])
    finally:
        plan.close()
    assert list(ev.factor_ranks) == rec["factor_ranks"]
    assert ev.info["factor_prec"] == rec["factor_prec"]
    assert ev.info["stored_factor_bytes"] == rec["stored_factor_bytes"]
    lls = [r["loglik"] for r in [rec] + rec["perturbed_1e-13"]]
    pad = 0.5 * (max(lls) - min(lls))
    print(f"case {q}: replayed decisions, loglik {ev.loglik:.6f} (reference {rec['loglik']:.6f})")
    assert min(lls) - pad <= ev.loglik <= max(lls) + pad


def test_mixed_rule_exact_where_no_entry_is_near_a_boundary(tlr):
    rec = _cases()[0]
    d = np.load(os.path.join(GOLD, rec["data"]))
    plan = tlr.get_plan(rec["n"], rec["b"])
    plan.set_precision("fp64")
    ev = plan.evaluate(rec["theta"], "mixed", rec["tau"], host_S=d["S"], host_y=d["y"])
    assert list(ev.factor_ranks) == rec["factor_ranks"]
    assert ev.info["factor_prec"] == rec["factor_prec"]
    assert ev.info["stored_factor_bytes"] == rec["stored_factor_bytes"]
    assert abs(ev.loglik - rec["loglik"]) <= EXACT_REL_TOL * abs(rec["loglik"]), (ev.loglik, rec["loglik"])


@pytest.mark.parametrize("q", range(len(_cases())))
def test_mixed_rule_within_reference_spread(tlr, q):
    rec = _cases()[q]
    d = np.load(os.path.join(GOLD, rec["data"]))
    bounds = tlr.tile_bounds(rec["n"], rec["b"])
    ll, fac, info = tlr.tlr_loglik(d["S"], d["y"], rec["theta"], bounds, "mixed", rec["tau"])
    runs = [rec] + rec["perturbed_1e-13"]
    lls = [r["loglik"] for r in runs]
    lo, hi = min(lls), max(lls)
    pad = 0.5 * (hi - lo)
    print(f"case {q}: loglik {ll:.6f}, reference spread [{lo:.6f}, {hi:.6f}]")
    assert lo - pad <= ll <= hi + pad
    assert abs(info["stored_factor_bytes"] - rec["stored_factor_bytes"]) <= 0.01 * rec["stored_factor_bytes"]
    for bits, cnt in rec["precision_mix_factor_tiles"].items():
        assert abs(info["precision_mix_factor_tiles"][int(bits)] - cnt) <= 5
    # the drop-in call surface carries the reference's info keys
    for key in ("stored_factor_bytes", "dense_factor_bytes", "factor_bytes_frac", "precision_mix_factor_tiles"):
        assert key in info
