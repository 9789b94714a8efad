"""Autotuner for batched evaluation: how many device workspaces (concurrent plans, one stream
each) a PlanBatch should run for a given problem.

More workspaces overlap more of the factorizations' latency-bound steps (the late steps with few
trailing pairs, the POTRF clusters, the backward pass's per-block-row launches), until the
recompression kernel saturates the GPU; each one holds a whole plan's memory (about 10 GB at
N = 50,000, b = 500).  tune_workspaces() times a short batched loglik+grad run for every
candidate that fits the device's free memory and records evals/s per candidate in a JSON table
keyed by (N, b, rule, value, precision); PlanBatch(..., workspaces="auto") reads the table and
takes the fastest entry for the nearest N with the same b, or falls back to min(count, 4).

No counterpart in the reference (it evaluates one parameter vector at a time).

Usage:  python -m adaptive_tlr_pilots_b200.autotune --n 50000 --b 500   (writes tuning.json)
        python -m adaptive_tlr_pilots_b200.autotune --n 50000 --b 250,500,1000 --candidates 4,8
        (one entry per tile size, each with its log-likelihood at theta_0 and its stored factor:
        tile_sizes() lists them; the tile size changes the approximation, so it is reported, not
        chosen silently)
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")
DEFAULT_WORKSPACES = 4


def _key(n, b, rule, value, precision):
    return f"n={int(n)} b={int(b)} rule={rule} value={float(value):g} precision={precision}"


def load_table(path=TABLE):
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return {}


def best_workspaces(n, b, count, rule="adaptive", value=0.9, precision="mixed", path=TABLE):
    """The fastest measured workspace count for the nearest tuned N with the same tile size, rule
    and precision, capped at `count`; min(count, DEFAULT_WORKSPACES) when nothing is tuned."""
    table = load_table(path)
    best, dist = None, None
    for entry in table.values():
        if (entry["b"], entry["rule"], entry["precision"]) != (int(b), rule, precision):
            continue
        if abs(entry["value"] - float(value)) > 1e-12:
            continue
        d = abs(np.log(entry["n"] / float(n)))
        if dist is None or d < dist:
            best, dist = entry, d
    if best is None:
        return max(1, min(int(count), DEFAULT_WORKSPACES))
    return max(1, min(int(count), int(best["best"])))


def tune_workspaces(S, y, b, candidates=(1, 2, 4, 6, 8), rule="adaptive", value=0.9, precision="mixed",
                    steps=2, device=0, path=TABLE, seed=20261021, per_plan_gb=None):
    """Time `steps` batched loglik+grad calls of w parameter vectors (theta_0 = (1, 0.3, 0.05) and
    seeded neighbours) through w workspaces for every candidate w that fits the free device memory;
    record {w: evals/s} and the fastest w in the table at `path`.  Returns the table entry."""
    import torch

    from .tlr import PlanBatch
    n = int(np.asarray(S).shape[0])
    rng = np.random.default_rng(seed)
    theta0 = np.array([1.0, 0.3, 0.05])
    rates = {}
    for w in candidates:
        free, _ = torch.cuda.mem_get_info(device)
        if per_plan_gb is not None and w * per_plan_gb * 1e9 > 0.9 * free:
            continue
        try:
            pb = PlanBatch(n, b, w, device=device, precision=precision)
        except RuntimeError:  # the workspaces did not fit
            torch.cuda.empty_cache()
            continue
        try:
            pb.set_data(S, y)
            thetas = theta0[None, :] * np.exp(0.05 * rng.standard_normal((w, 3)))
            pb.evaluate(thetas, rule, value)  # warm-up
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            for _ in range(steps):
                pb.evaluate(thetas, rule, value)
            torch.cuda.synchronize(device)
            rates[w] = w * steps / (time.perf_counter() - t0)
        except _lib.TlrError as e:  # a workspace's arena did not fit beside the others
            if e.code != _lib.ERR_NOMEM:
                raise
        finally:
            pb.close()
            torch.cuda.empty_cache()
    if not rates:
        raise RuntimeError("no workspace count fitted the device")
    # what the tile size does to the approximation at theta_0 (the tile size is the caller's
    # modelling choice: the table reports, it does not pick b)
    from .tlr import Plan
    plan = Plan(n, b, device=device)
    plan.set_precision(precision)
    plan.set_data(S, y)
    ev = plan.evaluate(theta0, rule, value)
    plan.close()
    torch.cuda.empty_cache()
    entry = dict(n=n, b=int(b), rule=rule, value=float(value), precision=precision,
                 evals_per_s={str(k): v for k, v in rates.items()}, best=int(max(rates, key=rates.get)),
                 gpu=torch.cuda.get_device_name(device), loglik_theta0=ev.loglik,
                 stored_factor=ev.info.get("stored_factor"), mean_rank_factor=ev.info.get("mean_rank_factor"),
                 max_rank_factor=ev.info.get("max_rank_factor"))
    table = load_table(path)
    table[_key(n, b, rule, value, precision)] = entry
    json.dump(table, open(path, "w"), indent=1, sort_keys=True)
    return entry


def tile_sizes(n, rule="adaptive", value=0.9, precision="mixed", path=TABLE):
    """{b: (best evals/s, loglik at theta_0, stored factor values)} of every tuned tile size at the
    nearest tuned N, for choosing b knowingly: b changes the approximation as well as the speed."""
    table = load_table(path)
    rows = [e for e in table.values() if e["rule"] == rule and e["precision"] == precision
            and abs(e["value"] - float(value)) <= 1e-12]
    if not rows:
        return {}
    n0 = min({e["n"] for e in rows}, key=lambda m: abs(np.log(m / float(n))))
    return {e["b"]: (max(e["evals_per_s"].values()), e.get("loglik_theta0"), e.get("stored_factor"))
            for e in rows if e["n"] == n0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=50000)
    ap.add_argument("--b", default="500", help="tile size, or several separated by commas")
    ap.add_argument("--tau", type=float, default=0.9)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--candidates", default="1,2,4,6,8")
    ap.add_argument("--steps", type=int, default=2)
    a = ap.parse_args()
    from . import synth
    S, y, _, _ = synth.simulate_field(a.n, (1.0, 0.3, 0.05))
    for b in (int(v) for v in a.b.split(",")):
        entry = tune_workspaces(S, y, b, candidates=tuple(int(c) for c in a.candidates.split(",")),
                                value=a.tau, precision=a.precision, steps=a.steps)
        print(json.dumps(entry), flush=True)


if __name__ == "__main__":
    main()
