"""The forward pass replayed from a CUDA graph computes exactly what its launches compute one by
one: the same log-likelihood, gradient, ranks, storage bits and failure verdicts, for every rule
and precision, with theta, the rule and the thresholds changing between replays of one captured
graph (they reach the kernels through the plan's device control block)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

THETAS = [[1.0, 0.3, 0.05], [1.4, 0.25, 0.08], [0.7, 0.4, 0.03]]
# (rule, value) in the order one plan meets them: the graph captured by the first serves the rest
RULES = [("adaptive", 0.9), ("fixed", 1e-4), ("mixed", 0.9), ("adaptive", 0.5), ("fixed", 1e-3)]


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


@pytest.fixture(scope="module")
def field():
    d = np.load(os.path.join(GOLD, "n4000_b250_data.npz"))
    return d["S"], d["y"]


def _plan(tlr, field, precision, graphs):
    S, y = field
    p = tlr.Plan(4000, 250)
    p.set_precision(precision)
    p.set_graphs(graphs)
    p.set_data(S, y)
    return p


def _same(a, b):
    assert a.status == b.status
    if a.status != 0:
        assert a.info["failed_at"] == b.info["failed_at"]
        return
    assert a.loglik == b.loglik
    assert np.array_equal(a.grad, b.grad)
    assert np.array_equal(a.sigma_ranks, b.sigma_ranks)
    assert np.array_equal(a.factor_ranks, b.factor_ranks)
    for key in ("stored_sigma", "stored_factor", "logdet", "quad"):
        assert a.info[key] == b.info[key], key
    if "factor_prec" in a.info:
        assert list(a.info["factor_prec"]) == list(b.info["factor_prec"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_equals_direct_launches(tlr, field, precision):
    g = _plan(tlr, field, precision, True)
    d = _plan(tlr, field, precision, False)
    failed = 0
    for rule, value in RULES:
        for th in THETAS:
            a = g.evaluate(th, rule, value, grad=True)
            b = d.evaluate(th, rule, value, grad=True)
            _same(a, b)
            failed += a.status != 0
    # fixed eps = 1e-3 fails on this field (diagonal tile 3 at the first theta): the replays after
    # a failing one start from a clean control block
    assert failed >= 1
    # the same number of kernel launches is counted either way
    lg = {k: v["launches"] for k, v in g.kernel_stats().items()}
    ld = {k: v["launches"] for k, v in d.kernel_stats().items()}
    assert lg == ld
    g.close()
    d.close()


def test_graph_with_rank_map_and_profiling(tlr, field):
    """Record, then replay the ranks at another theta, through the graph; profiling on issues the
    launches one by one and changes nothing."""
    g = _plan(tlr, field, "fp64", True)
    d = _plan(tlr, field, "fp64", False)
    for p in (g, d):
        p.rank_map("record")
        p.evaluate(THETAS[0], "adaptive", 0.9)
        p.rank_map("replay")
    a = g.evaluate(THETAS[1], "adaptive", 0.9, grad=True)
    b = d.evaluate(THETAS[1], "adaptive", 0.9, grad=True)
    _same(a, b)
    ranks = g.rank_map_get()
    assert np.array_equal(ranks[0], d.rank_map_get()[0])
    g.set_profiling(True)
    c = g.evaluate(THETAS[1], "adaptive", 0.9, grad=True)
    g.set_profiling(False)
    _same(a, c)
    g.rank_map("rule")
    d.rank_map("rule")
    _same(g.evaluate(THETAS[2], "mixed", 0.9), d.evaluate(THETAS[2], "mixed", 0.9))
    g.close()
    d.close()
