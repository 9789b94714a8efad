"""The block-row cyclic TLR factorization through the library (tlr_dist_*), with its ranks run in
lockstep on one GPU (blockrow.evaluate_lockstep: one partitioned plan per rank, the exchanges
device copies).  Every tile is computed by the same kernels as on one plan, so the result must be
the single plan's bit for bit: log-likelihood, log-determinant, quadratic form, initial and factor
ranks, stored sizes, and the failing tile when the factorization breaks down."""
import json
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


def _same(single, ranks):
    for ev in ranks:
        assert ev.status == single.status
        assert ev.info["completed"] == single.info["completed"]
        assert ev.info["stored_sigma"] == single.info["stored_sigma"]
        assert np.array_equal(ev.sigma_ranks, single.sigma_ranks)
        if single.status != 0:
            assert ev.info["failed_at"] == single.info["failed_at"]
            continue
        assert ev.loglik == single.loglik
        for key in ("logdet", "quad", "stored_factor", "max_rank_factor", "mean_rank_factor"):
            assert ev.info[key] == single.info[key], key
        assert np.array_equal(ev.factor_ranks, single.factor_ranks)


def _plans(tlr, n, b, world, S, y, cap=64):
    ps = []
    for _ in range(world):
        p = tlr.Plan(n, b, cap=cap)
        p.set_data(S, y)
        ps.append(p)
    return ps


@pytest.mark.parametrize("world", [2, 3, 5])
@pytest.mark.parametrize("rule,value", [("adaptive", 0.9), ("fixed", 1e-4), ("fixed", 1e-3)])
def test_lockstep_equals_single_plan(tlr, world, rule, value):
    from adaptive_tlr_pilots_b200 import blockrow
    d = np.load(os.path.join(GOLD, "n4000_b250_data.npz"))
    S, y = d["S"], d["y"]
    theta = (1.0, 0.3, 0.05)
    single = tlr.Plan(4000, 250)
    single.set_data(S, y)
    ref = single.evaluate(theta, rule, value)
    plans = _plans(tlr, 4000, 250, world, S, y)
    out = blockrow.evaluate_lockstep(plans, theta, rule, value)
    _same(ref, out)
    if rule == "fixed" and value == 1e-3:
        assert ref.status == 4  # the reference's verdict on this field: diagonal tile 3
    # a partitioned plan refuses the one-plan calls
    from adaptive_tlr_pilots_b200 import _lib
    with pytest.raises(_lib.TlrError):
        plans[0].evaluate(theta, rule, value)
    for p in plans + [single]:
        p.close()


def test_lockstep_at_n20000_and_capacity_growth(tlr):
    """N = 20,000, b = 500 (40 block rows) on 4 ranks, against the single plan and the reference's
    fixture; then plans of capacity 8 (adaptive ranks reach 18 on the N = 4,000 field) grow
    together and still agree."""
    from adaptive_tlr_pilots_b200 import blockrow
    g = json.load(open(os.path.join(GOLD, "golden_c2.json")))
    d = np.load(os.path.join(GOLD, g["data"]))
    rec = g["cases"][0]
    S, y = d["S"], d["y_" + rec["name"]]
    single = tlr.Plan(g["n"], g["b"])
    single.set_data(S, y)
    ref = single.evaluate(rec["theta"], g["rule"], g["value"])
    plans = _plans(tlr, g["n"], g["b"], 4, S, y)
    out = blockrow.evaluate_lockstep(plans, rec["theta"], g["rule"], g["value"])
    _same(ref, out)
    assert np.array_equal(out[0].sigma_ranks, np.asarray(rec["sigma_ranks"]))
    if rec["completed"]:
        assert np.array_equal(out[2].factor_ranks, np.asarray(rec["factor_ranks"]))
        assert abs(out[1].loglik - rec["loglik"]) <= 1e-10 * abs(rec["loglik"])
    for p in plans + [single]:
        p.close()
    d = np.load(os.path.join(GOLD, "n4000_b250_data.npz"))
    S, y = d["S"], d["y"]
    single = tlr.Plan(4000, 250)
    single.set_data(S, y)
    ref = single.evaluate((1.0, 0.3, 0.05), "adaptive", 0.9)
    plans = _plans(tlr, 4000, 250, 2, S, y, cap=8)
    out = blockrow.evaluate_lockstep(plans, (1.0, 0.3, 0.05), "adaptive", 0.9)
    assert all(p.cap > 8 for p in plans)
    _same(ref, out)
    for p in plans + [single]:
        p.close()


def test_lockstep_ragged_tiles_more_ranks_than_rows_and_matern52(tlr):
    """N = 1,030 with b = 100 (a last block row of 30 sites): 3 ranks, and 13 ranks (more ranks
    than the 11 block rows: two own nothing); then the Matern 5/2 kernel on 4 ranks."""
    from adaptive_tlr_pilots_b200 import blockrow
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    S, y = d["S"], d["y"]
    theta = (1.0, 0.3, 0.05)
    single = tlr.Plan(1030, 100)
    single.set_data(S, y)
    for world in (3, 13):
        ref = single.evaluate(theta, "adaptive", 0.9)
        plans = _plans(tlr, 1030, 100, world, S, y)
        _same(ref, blockrow.evaluate_lockstep(plans, theta, "adaptive", 0.9))
        for p in plans:
            p.close()
    single.set_kernel(2.5)
    ref = single.evaluate(theta, "fixed", 1e-6)
    plans = _plans(tlr, 1030, 100, 4, S, y)
    for p in plans:
        p.set_kernel(2.5)
    _same(ref, blockrow.evaluate_lockstep(plans, theta, "fixed", 1e-6))
    for p in plans + [single]:
        p.close()


def test_distributed_driver_over_nccl_single_rank(tlr):
    """evaluate_distributed through a real NCCL process group (one rank: broadcast,
    all_gather_into_tensor and all_reduce on the device buffers), against the single plan."""
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from adaptive_tlr_pilots_b200 import blockrow
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=120), device_id=torch.device("cuda", 0))
    try:
        d = np.load(os.path.join(GOLD, "n4000_b250_data.npz"))
        S, y = d["S"], d["y"]
        single = tlr.Plan(4000, 250)
        single.set_data(S, y)
        ref = single.evaluate((1.0, 0.3, 0.05), "adaptive", 0.9)
        plan = tlr.Plan(4000, 250)
        plan.set_data(S, y)
        ex = blockrow.TorchExchange()
        assert not ex.local and ex.world == 1
        _same(ref, [blockrow.evaluate_distributed(plan, (1.0, 0.3, 0.05), "adaptive", 0.9)])
        plan.close()
        single.close()
    finally:
        dist.destroy_process_group()


def test_lockstep_plans_on_their_own_streams(tlr):
    """Ranks whose plans were created on different streams: the exchanges are fenced by
    device-wide synchronisations, and the result is still the single plan's."""
    import torch

    from adaptive_tlr_pilots_b200 import blockrow
    d = np.load(os.path.join(GOLD, "n4000_b250_data.npz"))
    S, y = d["S"], d["y"]
    single = tlr.Plan(4000, 250)
    single.set_data(S, y)
    ref = single.evaluate((1.0, 0.3, 0.05), "adaptive", 0.9)
    plans = []
    for _ in range(3):
        with torch.cuda.stream(torch.cuda.Stream()):
            p = tlr.Plan(4000, 250)
            p.set_data(S, y)
        plans.append(p)
    torch.cuda.synchronize()
    assert len({p.stream for p in plans}) == 3
    _same(ref, blockrow.evaluate_lockstep(plans, (1.0, 0.3, 0.05), "adaptive", 0.9))
    for p in plans + [single]:
        p.close()
