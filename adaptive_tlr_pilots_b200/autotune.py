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
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

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
        finally:
            pb.close()
            torch.cuda.empty_cache()
    if not rates:
        raise RuntimeError("no workspace count fitted the device")
    entry = dict(n=n, b=int(b), rule=rule, value=float(value), precision=precision,
                 evals_per_s={str(k): v for k, v in rates.items()}, best=int(max(rates, key=rates.get)),
                 gpu=torch.cuda.get_device_name(device))
    table = load_table(path)
    table[_key(n, b, rule, value, precision)] = entry
    json.dump(table, open(path, "w"), indent=1, sort_keys=True)
    return entry


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=50000)
    ap.add_argument("--b", type=int, default=500)
    ap.add_argument("--tau", type=float, default=0.9)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--candidates", default="1,2,4,6,8")
    ap.add_argument("--steps", type=int, default=2)
    a = ap.parse_args()
    from . import synth
    S, y, _, _ = synth.simulate_field(a.n, (1.0, 0.3, 0.05))
    entry = tune_workspaces(S, y, a.b, candidates=tuple(int(c) for c in a.candidates.split(",")),
                            value=a.tau, precision=a.precision, steps=a.steps)
    print(json.dumps(entry))


if __name__ == "__main__":
    main()
