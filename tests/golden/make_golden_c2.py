"""Generate the N = 20,000, b = 500 fixtures (the range x nugget sweep) by running the reference.

The reference's modules codes/11_tlr_rank_rules.py and codes/17_tlr_cholesky_pilot.py are
imported by file path, as its own scripts import each other (codes/17_tlr_cholesky_pilot.py:85-87).
Each field is simulated with its own theta by the reference's data protocol
(codes/17_tlr_cholesky_pilot.py:313-325, the --range / --eta flags of 17:300-301): seed 20261020,
N + 300 uniform sites, y = L z with L the dense FP64 Cholesky, a random split, Morton order.  The
sites depend only on the seed, so they are stored once; y is stored per case.

Per case the fixture holds the dense log-likelihood (11:112-120), and for the adaptive rule
tau = 0.9 the reference's tlr_loglik outputs (17:259-266): log-likelihood, log-determinant,
completion, stored values, every factor rank in the reference's L_off order, and every initial
(Sigma-tile) rank from its truncate_svd (17:107-116).

Usage:  python tests/golden/make_golden_c2.py [--ref /root/reference]   (about 15 min on 8 cores)
"""
import argparse
import json
import os
import time

import numpy as np

from make_golden import load, protocol, sigma_ranks

HERE = os.path.dirname(os.path.abspath(__file__))
N, B = 20000, 500
RANGES = (0.1, 0.3, 1.0)
ETAS = (0.05, 0.005)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    rules = load(a.ref, "rules", "11_tlr_rank_rules.py")
    tlr = load(a.ref, "tlr", "17_tlr_cholesky_pilot.py")
    gold = dict(source="reference codes/11_tlr_rank_rules.py + codes/17_tlr_cholesky_pilot.py, run by "
                       "make_golden_c2.py", n=N, b=B, rule="adaptive", value=0.9, data="n20000_b500_data.npz",
                cases=[])
    S0 = None
    ys = {}
    for rg in RANGES:
        for eta in ETAS:
            t0 = time.time()
            theta = (1.0, rg, eta)
            S, y = protocol(rules, N, theta)
            if S0 is None:
                S0 = S
            assert np.array_equal(S, S0), "the sites must not depend on theta"
            K = rules.cov_full(S, np.asarray(theta, float))
            ll_dense, _ = rules.loglik_dense(K, y)
            del K
            bounds = rules.tile_bounds(N, B)
            ll, fac, info = tlr.tlr_loglik(S, y, np.asarray(theta, float), bounds, "adaptive", 0.9)
            key = f"r{rg}_e{eta}"
            rec = dict(name=key, theta=list(theta), dense_loglik=float(ll_dense), completed=bool(info["completed"]),
                       stored_sigma=int(info["stored_sigma"]), max_rank_sigma=int(info["max_rank_sigma"]))
            if info["completed"]:
                L_diag, L_off = fac
                rec.update(loglik=float(ll), stored_factor=int(info["stored_factor"]),
                           mean_rank_factor=float(info["mean_rank_factor"]),
                           max_rank_factor=int(info["max_rank_factor"]),
                           logdet=float(2.0 * sum(np.log(np.diag(d)).sum() for d in L_diag)),
                           factor_ranks=[int(u.shape[1]) for u, _ in L_off.values()],
                           factor_keys=[list(k) for k in L_off.keys()])
                del fac, L_diag, L_off
            else:
                rec.update(failed_at=int(info["failed_at"]))
            rec["sigma_ranks"] = sigma_ranks(tlr, rules, S, B, theta, "adaptive", 0.9)
            ys[key] = y
            gold["cases"].append(rec)
            print(key, "dense", ll_dense, "tlr", rec.get("loglik"), rec.get("failed_at"),
                  f"{time.time() - t0:.0f}s", flush=True)
            json.dump(gold, open(os.path.join(HERE, "golden_c2.json"), "w"), indent=1)
    np.savez(os.path.join(HERE, gold["data"]), S=S0, **{"y_" + k: v for k, v in ys.items()})
    print("wrote", os.path.join(HERE, "golden_c2.json"))


if __name__ == "__main__":
    main()
