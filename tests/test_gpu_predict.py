"""Kriging prediction and products with the device factor (tlr_factor_solve, tlr_factor_matvec)
against the reference's own outputs (fixture from tests/golden/make_golden_predict.py)."""
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


def test_predict_matvec_and_solves_match_reference(tlr):
    import torch
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    f = np.load(os.path.join(GOLD, "predict_n1030.npz"))
    S, y = d["S"], d["y"]
    theta = (1.0, 0.3, 0.05)
    bounds = tlr.tile_bounds(len(y), 100)
    ll, fac, _ = tlr.tlr_loglik(S, y, theta, bounds, "adaptive", 0.9)
    assert abs(ll - float(f["loglik"])) <= 1e-10 * abs(ll)
    mu, sd = tlr.tlr_predict(S, y, f["Sp"], theta, bounds, fac)
    np.testing.assert_allclose(mu, f["mu"], rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(sd, f["sd"], rtol=1e-9)
    np.testing.assert_allclose(fac.matvec(torch.from_numpy(f["z"])).cpu().numpy(), f["Lz"], rtol=1e-9, atol=1e-11)
    fwd = fac.forward(torch.from_numpy(y)).cpu().numpy()
    np.testing.assert_allclose(fwd, f["fwd"], rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(fac.backward(torch.from_numpy(fwd)).cpu().numpy(), f["bwd"], rtol=1e-9, atol=1e-11)
    sk = tlr.skill(f["yp"], mu, sd)
    assert abs(sk["rmse"] - float(f["rmse"])) <= 1e-9 and abs(sk["crps"] - float(f["crps"])) <= 1e-9
    # multi-column solve: L^-1 [y, 2y] = [L^-1 y, 2 L^-1 y]
    two = fac.forward(torch.from_numpy(np.stack([y, 2 * y], 1))).cpu().numpy()
    np.testing.assert_allclose(two[:, 1], 2 * two[:, 0], rtol=1e-12, atol=1e-12)


def test_solve_needs_a_completed_factorization(tlr):
    """A plan whose last evaluation failed (not PD) refuses solves instead of using stale tiles."""
    d = np.load(os.path.join(GOLD, "n4000_b250_data.npz"))
    p = tlr.Plan(4000, 250)
    p.set_data(d["S"], d["y"])
    assert p.evaluate((1.0, 0.3, 0.05), "fixed", 1e-3).status == 4
    with pytest.raises(tlr._lib.TlrError):
        p.solve(np.ones(4000))
    p.close()
