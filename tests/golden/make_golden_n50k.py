"""Generate the N = 50,000, b = 500 rank fixture by running the reference itself.

The ranks of the TLR factorization depend only on the sites and theta, not on y, so the field is not
simulated: the sites are drawn by the reference's data protocol (codes/17_tlr_cholesky_pilot.py:
313-325 with seed 20261020: N + 300 uniform sites, the field's standard normals drawn and discarded,
the random split, Morton order by codes/11_tlr_rank_rules.py:40-53), and the reference's
tlr_cholesky (17:137-215) runs at theta = (1, 0.3, 0.05), adaptive tau = 0.9.  The fixture holds
every factor rank in the reference's L_off order, every initial (Sigma-tile) rank in the order
(i, j < i) from its truncate_svd (17:107-116), and the stored values.  About 7 minutes on 8 cores.

Usage:  python tests/golden/make_golden_n50k.py [--ref /root/reference]
"""
import argparse
import json
import os

import numpy as np

from make_golden import load

HERE = os.path.dirname(os.path.abspath(__file__))
N, B, N_PRED, SEED = 50000, 500, 300, 20261020


def sites(rules):
    rng = np.random.default_rng(SEED)
    S_all = rng.random((N + N_PRED, 2))
    rng.standard_normal(N + N_PRED)  # the field's normals (17:316), drawn to keep the stream in step
    perm = rng.permutation(N + N_PRED)
    S = S_all[perm[:N]]
    return S[rules.morton_order(S)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    rules = load(a.ref, "rules", "11_tlr_rank_rules.py")
    tlr = load(a.ref, "tlr", "17_tlr_cholesky_pilot.py")
    S = sites(rules)
    theta = np.array([1.0, 0.3, 0.05])
    bounds = rules.tile_bounds(N, B)
    thr_abs = 0.9 * B * theta[0] * theta[2] / N
    sigma_ranks = []
    for i, (i0, i1) in enumerate(bounds):  # the initial ranks, as 17:159-165 computes them
        for j, (j0, j1) in enumerate(bounds[:i]):
            T = theta[0] * rules.matern32(rules.dist(S[i0:i1], S[j0:j1]), theta[1])
            U, V, _ = tlr.truncate_svd(T, "adaptive", None, thr_abs)
            sigma_ranks.append(int(U.shape[1]))
    L_diag, L_off, info = tlr.tlr_cholesky(S, theta, bounds, "adaptive", 0.9)
    out = dict(source="reference codes/11_tlr_rank_rules.py + codes/17_tlr_cholesky_pilot.py, run by "
                      "make_golden_n50k.py", n=N, b=B, seed=SEED, theta=theta.tolist(), rule="adaptive", value=0.9,
               completed=bool(info["completed"]), stored_sigma=int(info["stored_sigma"]),
               max_rank_sigma=int(info["max_rank_sigma"]), stored_factor=int(info["stored_factor"]),
               mean_rank_factor=float(info["mean_rank_factor"]), max_rank_factor=int(info["max_rank_factor"]),
               sigma_ranks=sigma_ranks, factor_ranks=[int(u.shape[1]) for u, _ in L_off.values()])
    json.dump(out, open(os.path.join(HERE, "golden_n50k.json"), "w"))
    print("stored_factor", out["stored_factor"], "mean", out["mean_rank_factor"], "max", out["max_rank_factor"])


if __name__ == "__main__":
    main()
