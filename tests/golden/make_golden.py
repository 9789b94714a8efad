"""Generate the golden fixtures under tests/golden/ by running the reference itself.

The reference (marysalvana/adaptive-tlr-pilots) is plain Python; its modules
codes/11_tlr_rank_rules.py and codes/17_tlr_cholesky_pilot.py are imported by file path,
exactly as its own scripts import each other (codes/17_tlr_cholesky_pilot.py:85-87), and
run on seeded inputs built with the reference's own data protocol
(codes/17_tlr_cholesky_pilot.py:313-325).  The outputs are written as small JSON/NPZ
fixtures so that tests can run where the reference is absent.

Usage:  python tests/golden/make_golden.py [--ref /root/reference]
"""
import argparse
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load(ref, name, fname):
    spec = importlib.util.spec_from_file_location(name, os.path.join(ref, "codes", fname))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def protocol(rules, n, theta, seed=20261020, n_pred=300):
    # the reference's data protocol, codes/17_tlr_cholesky_pilot.py:313-325
    rng = np.random.default_rng(seed)
    theta = np.asarray(theta, float)
    n_tot = n + n_pred
    S_all = rng.random((n_tot, 2))
    L = np.linalg.cholesky(rules.cov_full(S_all, theta))
    y_all = L @ rng.standard_normal(n_tot)
    perm = rng.permutation(n_tot)
    obs = perm[:n]
    S, y = S_all[obs], y_all[obs]
    order = rules.morton_order(S)
    return S[order], y[order]


def run_rules(tlr, rules, S, y, b, theta, specs):
    bounds = rules.tile_bounds(len(y), b)
    out = []
    for rule, value in specs:
        ll, fac, info = tlr.tlr_loglik(S, y, np.asarray(theta, float), bounds, rule, value)
        rec = dict(rule=rule, value=value, completed=bool(info["completed"]),
                   stored_sigma=int(info["stored_sigma"]), max_rank_sigma=int(info["max_rank_sigma"]))
        if info["completed"]:
            L_diag, L_off = fac
            rec.update(loglik=ll, stored_factor=int(info["stored_factor"]),
                       mean_rank_factor=float(info["mean_rank_factor"]),
                       max_rank_factor=int(info["max_rank_factor"]),
                       factor_ranks=[int(u.shape[1]) for u, _ in L_off.values()],
                       factor_keys=[list(k) for k in L_off.keys()],
                       logdet=float(2.0 * sum(np.log(np.diag(d)).sum() for d in L_diag)))
        else:
            rec.update(failed_at=int(info["failed_at"]))
        out.append(rec)
    return out


def sigma_ranks(tlr, rules, S, b, theta, rule, value):
    """Initial (Sigma-tile) ranks in the order (i, j<i), from the reference's truncate_svd."""
    n = S.shape[0]
    bounds = rules.tile_bounds(n, b)
    bmax = max(e - s for s, e in bounds)
    sigma2, r, eta = theta
    thr_rel = value if rule == "fixed" else None
    thr_abs = value * bmax * sigma2 * eta / n if rule == "adaptive" else None
    ranks = []
    for i, (i0, i1) in enumerate(bounds):
        for j, (j0, j1) in enumerate(bounds[:i]):
            T = sigma2 * rules.matern32(rules.dist(S[i0:i1], S[j0:j1]), r)
            U, V, _ = tlr.truncate_svd(T, rule, thr_rel, thr_abs)
            ranks.append(int(U.shape[1]))
    return ranks


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    rules = load(a.ref, "rules", "11_tlr_rank_rules.py")
    tlr = load(a.ref, "tlr", "17_tlr_cholesky_pilot.py")
    theta = (1.0, 0.3, 0.05)
    gold = dict(source="reference codes/11_tlr_rank_rules.py + codes/17_tlr_cholesky_pilot.py, run by make_golden.py",
                cases=[])

    # 1. Morton order, including duplicates, boundary values and out-of-square points
    rng = np.random.default_rng(7)
    xy = rng.random((500, 2))
    xy[10] = xy[20]; xy[30] = xy[20]
    xy[40] = [0.0, 0.0]; xy[41] = [1.0, 1.0]; xy[42] = [-0.25, 1.5]; xy[43] = [0.9999999, 0.0]
    xy[44:60] = np.round(xy[44:60] * 8) / 8
    np.savez(os.path.join(HERE, "morton_case.npz"), xy=xy, perm=rules.morton_order(xy))

    # 2. dense and TLR log-likelihoods on the N = 4,000, b = 250 field (adaptive tau = 0.9, fixed
    #    eps = 1e-3 and 1e-4) and on smaller / ragged cases
    configs = [
        dict(name="n4000_b250", n=4000, b=250, theta=theta,
             specs=[("adaptive", 0.9), ("fixed", 1e-3), ("fixed", 1e-4)], save_data=True),
        dict(name="n1030_b100", n=1030, b=100, theta=theta,
             specs=[("adaptive", 0.9), ("fixed", 1e-4), ("fixed", 1e-2)], save_data=True),
        dict(name="n2000_b200_r1.0_e0.005", n=2000, b=200, theta=(1.0, 1.0, 0.005),
             specs=[("adaptive", 0.9), ("fixed", 1e-5)], save_data=True),
        dict(name="n1500_b250_s2.5_r0.1", n=1500, b=250, theta=(2.5, 0.1, 0.2),
             specs=[("adaptive", 0.5), ("fixed", 1e-3)], save_data=True),
    ]
    for cfg in configs:
        S, y = protocol(rules, cfg["n"], cfg["theta"])
        K = rules.cov_full(S, np.asarray(cfg["theta"], float))
        ll_dense, _ = rules.loglik_dense(K, y)
        del K
        res = run_rules(tlr, rules, S, y, cfg["b"], cfg["theta"], cfg["specs"])
        for rec in res:
            rec["sigma_ranks"] = sigma_ranks(tlr, rules, S, cfg["b"], cfg["theta"], rec["rule"], rec["value"])
        case = dict(name=cfg["name"], n=cfg["n"], b=cfg["b"], theta=list(cfg["theta"]),
                    dense_loglik=float(ll_dense), rules=res, data=f"{cfg['name']}_data.npz")
        np.savez(os.path.join(HERE, case["data"]), S=S, y=y)
        gold["cases"].append(case)
        print(cfg["name"], "dense", ll_dense, [(r["rule"], r["value"], r.get("loglik"), r.get("failed_at")) for r in res],
              flush=True)

    # 3. values the reference itself committed (results/tlr_cholesky/tlr_cholesky_n10000.json)
    committed = json.load(open(os.path.join(a.ref, "results", "tlr_cholesky", "tlr_cholesky_n10000.json")))
    gold["committed_n10000"] = dict(
        source="results/tlr_cholesky/tlr_cholesky_n10000.json (on results/tlr_cholesky/sim_n10000_obs.csv)",
        dense_loglik=committed["dense_loglik_true"],
        rules=[{k: r.get(k) for k in ("rule", "value", "completed", "failed_at_tile", "stored_sigma", "stored_factor",
                                      "mean_rank_factor", "max_rank_factor", "loglik_err")}
               for r in committed["rules"]])
    json.dump(gold, open(os.path.join(HERE, "golden.json"), "w"), indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
