"""Golden fixtures for the Matern 5/2 kernel, made by running the reference itself.

codes/24_screening_stress.py is imported by file path; its set_kernel(2.5) replaces the kernel of
the TLR Cholesky of codes/17_tlr_cholesky_pilot.py (24:46-47), exactly as its regime sweeps do.
The reference's tlr_loglik then runs on the sites and observations of two existing fixtures
(n1030_b100, n4000_b250) for three rules; ranks, stored values, log-likelihoods and the dense
FP64 log-likelihood go to golden_nu52.json.

Usage:  python tests/golden/make_golden_nu52.py [--ref /root/reference]
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import load, run_rules, sigma_ranks  # noqa: E402

CASES = [("n1030_b100", "n1030_b100_data.npz", 100, (1.0, 0.3, 0.05)),
         ("n4000_b250", "n4000_b250_data.npz", 250, (1.0, 0.3, 0.05))]
SPECS = [("adaptive", 0.9), ("fixed", 1e-4), ("fixed", 1e-6)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    m24 = load(a.ref, "screening_stress", "24_screening_stress.py")
    m24.set_kernel(2.5)
    tlr, rules = m24.tlr, m24.rules
    out = []
    for name, data, b, theta in CASES:
        d = np.load(os.path.join(HERE, data))
        S, y = d["S"], d["y"]
        recs = run_rules(tlr, rules, S, y, b, theta, SPECS)
        for rec in recs:
            rec["sigma_ranks"] = sigma_ranks(tlr, rules, S, b, theta, rec["rule"], rec["value"])
        dense, _ = rules.loglik_dense(rules.cov_full(S, np.asarray(theta, float)), y)
        out.append(dict(name=name, data=data, n=int(len(y)), b=b, theta=list(theta), nu=2.5,
                        dense_loglik=float(dense), rules=recs))
        print(name, [(r["rule"], r["value"], r.get("loglik"), r.get("max_rank_factor")) for r in recs], flush=True)
    with open(os.path.join(HERE, "golden_nu52.json"), "w") as f:
        json.dump(dict(source="codes/24_screening_stress.py set_kernel(2.5) + codes/17_tlr_cholesky_pilot.py tlr_loglik",
                       cases=out), f)


if __name__ == "__main__":
    main()
