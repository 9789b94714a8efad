"""Generate the assembled-matrix-rule fixtures by running the reference itself.

Runs, on the N = 4,000, b = 250 golden field (tests/golden/n4000_b250_data.npz, made by
make_golden.py with the reference's data protocol), for the rules adaptive tau = 0.9, fixed
eps = 1e-3 and fixed eps = 1e-4 at theta = (1, 0.3, 0.05):

  * codes/11_tlr_rank_rules.py make_cov / truncate_tiles (11:74-108, 121-126) and loglik_dense
    (11:112-120): stored values, max relative / absolute tile error, ||Sigma - Sigma^TLR||_F,
    every tile rank, and the dense log-likelihood of Sigma^TLR;
  * codes/19_tlr_mcmc_gpu.py Likelihood (19:27-138) on torch's CPU device, svd_mode fp64, fp32
    and rand: the log-likelihood and stored values.

The modules are imported by file path, as the reference's scripts import each other.

Usage:  python tests/golden/make_golden_assembled.py [--ref /root/reference]
"""
import argparse
import json
import os

import numpy as np

from make_golden import load

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    rules = load(a.ref, "rules", "11_tlr_rank_rules.py")
    mc = load(a.ref, "mcmc_gpu", "19_tlr_mcmc_gpu.py")
    import torch
    d = np.load(os.path.join(HERE, "n4000_b250_data.npz"))
    S, y = d["S"], d["y"]
    n, b = len(y), 250
    theta = np.array([1.0, 0.3, 0.05])
    bounds = rules.tile_bounds(n, b)
    out = dict(source="reference codes/11_tlr_rank_rules.py and codes/19_tlr_mcmc_gpu.py, run by "
                      "make_golden_assembled.py", data="n4000_b250_data.npz", n=n, b=b, theta=theta.tolist(),
               rules=[])
    like = {m: mc.Likelihood(S, y, b, torch.device("cpu"), svd_mode=m) for m in ("fp64", "fp32", "rand")}
    for rule, value in [("adaptive", 0.9), ("fixed", 1e-3), ("fixed", 1e-4)]:
        K, info = rules.make_cov(S, theta, rule, value, bounds)
        stored, max_rel, max_abs, fro, ranks = info
        ll, _ = rules.loglik_dense(K, y)
        rec = dict(rule=rule, value=value, stored=int(stored), max_rel=float(max_rel), max_abs=float(max_abs),
                   fro_err=float(fro), ranks=[int(r) for r in ranks], loglik=None if ll is None else float(ll),
                   likelihood19={})
        for m, L in like.items():
            v = L(theta, rule, value)
            rec["likelihood19"][m] = dict(loglik=float(v), ok=bool(L.last["ok"]), stored=int(L.last["stored"]))
        out["rules"].append(rec)
        print(rule, value, stored, ll, {m: r["loglik"] for m, r in rec["likelihood19"].items()}, flush=True)
    json.dump(out, open(os.path.join(HERE, "golden_assembled.json"), "w"), indent=1)
    print("wrote", os.path.join(HERE, "golden_assembled.json"))


if __name__ == "__main__":
    main()
