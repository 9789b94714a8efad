"""Generate fixtures of the reference's storage-precision rule 'mixed' by running it.

codes/17_tlr_cholesky_pilot.py with rule = "mixed" (17:33-82, used at 17:146-148, 163-164,
183-184, 203-204, 210-214): the adaptive rank rule, and every stored factor pair rounded to the
lowest of FP8 (E4M3-like), FP16, FP32, FP64 whose rounding error fits the budget left after
truncation.  Run on the golden fields of make_golden.py (N = 1,030 / b = 100 and N = 4,000 /
b = 250, theta = (1, 0.3, 0.05)), the module imported by file path as the reference's scripts do.
Per case: log-likelihood, log-determinant, completion, factor ranks and the precision of every
factor tile in the reference's L_off order, stored values and bytes, the precision mix.

The rule is ill-conditioned in its inputs: a pair stored in FP16 turns a difference of 1e-13 in
one factor entry into a jump of 2^-11 whenever the entry lies near a rounding boundary, and many
of the rule's rank and storage decisions sit within a few percent of their budgets.  So every case
also records the reference's own spread: the same rule on the sites multiplied by
(1 + 1e-13 z), z standard normal, for eight seeds (log-likelihood, stored bytes, precision mix).

Usage:  python tests/golden/make_golden_mixed_rule.py [--ref /root/reference]
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
    tlr = load(a.ref, "tlr", "17_tlr_cholesky_pilot.py")
    out = dict(source="reference codes/17_tlr_cholesky_pilot.py rule 'mixed', run by make_golden_mixed_rule.py",
               cases=[])
    for data, b, tau in [("n1030_b100_data.npz", 100, 0.9), ("n4000_b250_data.npz", 250, 0.9),
                         ("n4000_b250_data.npz", 250, 0.5)]:
        d = np.load(os.path.join(HERE, data))
        S, y = d["S"], d["y"]
        theta = np.array([1.0, 0.3, 0.05])
        bounds = rules.tile_bounds(len(y), b)
        ll, fac, info = tlr.tlr_loglik(S, y, theta, bounds, "mixed", tau)
        rec = dict(data=data, n=len(y), b=b, theta=theta.tolist(), tau=tau, completed=bool(info["completed"]),
                   stored_sigma=int(info["stored_sigma"]))
        if info["completed"]:
            L_diag, L_off = fac
            rec.update(loglik=float(ll), logdet=float(2.0 * sum(np.log(np.diag(dd)).sum() for dd in L_diag)),
                       stored_factor=int(info["stored_factor"]), stored_factor_bytes=int(info["stored_factor_bytes"]),
                       factor_bytes_frac=float(info["factor_bytes_frac"]),
                       precision_mix_factor_tiles={str(k): int(v) for k, v in info["precision_mix_factor_tiles"].items()},
                       factor_ranks=[int(u.shape[1]) for u, _ in L_off.values()],
                       factor_prec=[int(tlr.PREC_OF[k]) for k in L_off.keys()])
        else:
            rec.update(failed_at=int(info["failed_at"]))
        spread = []
        for seed in range(8):
            Sp = S * (1.0 + 1e-13 * np.random.default_rng(seed).standard_normal(S.shape))
            llp, _, infop = tlr.tlr_loglik(Sp, y, theta, bounds, "mixed", tau)
            spread.append(dict(seed=seed, completed=bool(infop["completed"]),
                               loglik=None if llp is None else float(llp),
                               stored_factor_bytes=int(infop.get("stored_factor_bytes", 0)),
                               precision_mix_factor_tiles={str(k): int(v) for k, v in
                                                           infop.get("precision_mix_factor_tiles", {}).items()}))
        rec["perturbed_1e-13"] = spread
        out["cases"].append(rec)
        print(data, tau, rec.get("loglik"), rec.get("precision_mix_factor_tiles"), flush=True)
    json.dump(out, open(os.path.join(HERE, "golden_mixed_rule.json"), "w"), indent=1)
    print("wrote", os.path.join(HERE, "golden_mixed_rule.json"))


if __name__ == "__main__":
    main()
