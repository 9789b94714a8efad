"""Golden fixture for kriging prediction and the factor product, made by running the reference.

Imports codes/11_tlr_rank_rules.py and codes/17_tlr_cholesky_pilot.py by file path (as the
reference's scripts do), factors the N = 1,030 golden field (n1030_b100_data.npz) with the
adaptive rule tau = 0.9 at theta = (1, 0.3, 0.05), and records tlr_predict (17:269-276) at 60
seeded prediction sites, tlr_matvec_L (17:218-227) of a seeded standard normal vector, the
reference's skill scores (11:162-165) of the prediction against seeded "held-out" values, and
tlr_forward / tlr_backward (17:230-256) of the observations.

Usage:  python tests/golden/make_golden_predict.py [--ref /root/reference]
"""
import argparse
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load(ref, name, fname):
    spec = importlib.util.spec_from_file_location(name, os.path.join(ref, "codes", fname))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    rules = load(a.ref, "rules", "11_tlr_rank_rules.py")
    tlr = load(a.ref, "tlr", "17_tlr_cholesky_pilot.py")
    d = np.load(os.path.join(HERE, "n1030_b100_data.npz"))
    S, y = d["S"], d["y"]
    theta = np.array([1.0, 0.3, 0.05])
    bounds = rules.tile_bounds(len(y), 100)
    ll, fac, info = tlr.tlr_loglik(S, y, theta, bounds, "adaptive", 0.9)
    rng = np.random.default_rng(20261022)
    Sp = rng.random((60, 2))
    z = rng.standard_normal(len(y))
    mu, sd = tlr.tlr_predict(S, y, Sp, theta, bounds, fac)
    yp = mu + sd * rng.standard_normal(60)
    sk = rules.skill(yp, mu, sd)
    Lz = tlr.tlr_matvec_L(fac[0], fac[1], bounds, z[:, None])[:, 0]
    fwd = tlr.tlr_forward(fac[0], fac[1], bounds, y[:, None])[:, 0]
    bwd = tlr.tlr_backward(fac[0], fac[1], bounds, fwd[:, None])[:, 0]
    np.savez(os.path.join(HERE, "predict_n1030.npz"), Sp=Sp, mu=mu, sd=sd, yp=yp, z=z, Lz=Lz, fwd=fwd, bwd=bwd,
             rmse=sk["rmse"], crps=sk["crps"], cover90=sk["cover90"], loglik=ll)
    print("wrote predict_n1030.npz", ll, sk)


if __name__ == "__main__":
    main()
