#!/usr/bin/env python
"""Benchmark of the TLR Gaussian-process log-likelihood on B200.

Workload: N = 50,000 seeded sites (the reference's data protocol, codes/17_tlr_cholesky_pilot.py:
313-325), Morton-ordered, tiles b = 500, Matern-3/2 at theta = (1, 0.3, 0.05), adaptive rule
tau = 0.9; one step = one log-likelihood + gradient evaluation (tile generation, compression, TLR
Cholesky, solve, selected-inversion backward, dSigma contraction) on the plain FP64 path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (launched by torch.distributed.run) every rank evaluates its own replica of the
workload (independent evaluations, no collective on the data path: weak scaling); the device time
is the max over ranks.  --impl reference times the reference pipeline on the host's cores
(the CPU oracle, a restatement of codes/17_tlr_cholesky_pilot.py) on a bounded sample.
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

THETA = (1.0, 0.3, 0.05)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=50000)
    ap.add_argument("--b", type=int, default=500)
    ap.add_argument("--tau", type=float, default=0.9)
    ap.add_argument("--cpu-sample", type=int, default=1, help="0: skip the CPU baseline leg")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--plain-steps", type=int, default=-1,
                    help="timed evaluations of the plain FP64 comparison (-1: as many as the batched leg, steps x "
                         "batch; 0: skip)")
    ap.add_argument("--batch", type=int, default=8,
                    help="parameter vectors per step (one batched call, one workspace each: the autotuner's best "
                         "at N=50k, b=500)")
    ap.add_argument("--dense", type=int, default=1, help="0: skip the dense FP64 oracle")
    ap.add_argument("--sim", choices=["dense", "tlr"], default="dense",
                    help="field from a dense Cholesky, or from a tau = 0.02 TLR factor (large N)")
    ap.add_argument("--chains", type=int, default=0,
                    help="> 0: instead of the headline, run this many lockstep random-walk chains (the 64-chain "
                         "configuration) for --chain-iters iterations through --workspaces device workspaces")
    ap.add_argument("--workspaces", type=int, default=8)
    ap.add_argument("--blockrow", type=int, default=0,
                    help="1: one log-likelihood split over the ranks, block rows cyclic (strong scaling)")
    ap.add_argument("--graphs", type=int, default=1,
                    help="1: forward pass replayed from a CUDA graph (the library default); 0: launches one by one")
    ap.add_argument("--chain-iters", type=int, default=3)
    return ap.parse_args()


# k_recompress DRAM traffic per launch at N = 50,000, b = 500, adaptive tau = 0.9 (bytes): the mean of
# dram__bytes_read.sum + dram__bytes_write.sum over the 98 launches of one evaluation, from an ncu
# capture of `bench.py --steps 1 --warmup 1 --cpu-sample 0 --plain-steps 0 --batch 1 --dense 0 --graphs 0`
# (the same kernels launched one by one: ncu's driver reported a failed launch replaying the graph)
RC_TRAFFIC_N50K = 205.8e6
RC_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, mean over the 98 k_recompress launches of "
                     "one evaluation (batch 1, same workload, launches one by one, 1-pass capture)")
METRIC = "TLR loglik+grad evals/s at N=50k vs plain FP64 on B200; |dl| vs FP64 dense"


def workload(a):
    return {"workload": f"TLR log-likelihood, N={a.n}, b={a.b}, Matern-3/2 theta=(1,0.3,0.05), adaptive tau={a.tau}",
            "n": a.n, "b": a.b, "rule": "adaptive", "tau": a.tau, "precision": a.precision,
            "theta_per_step": a.batch, "batch": "theta_0 = (1, 0.3, 0.05), the others theta_0 exp(0.05 z), seeded",
            "l2": "inputs larger than L2 (per-evaluation working set several GB)",
            "forward": "CUDA graph replay" if a.graphs else "launches one by one"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_baseline(S, y, a):
    from oracle.cpu_sample import SampledPipeline, blas_threads
    t0 = time.perf_counter()
    sp = SampledPipeline(S, y, THETA, a.b, "adaptive", a.tau, n_pairs=48)
    setup = time.perf_counter() - t0
    est, wall = 0.0, 0.0
    for rep in range(4):
        e, w = sp.step(n_compress=24, n_trsm=32, n_recompress=96, seed=rep)
        est += e / 4
        wall += w
    return {"value": 1.0 / (7.0 * est), "unit": "evals/s", "cores": blas_threads(), "kind": "port",
            "sample": (f"oracle (NumPy/SciPy restatement of codes/17_tlr_cholesky_pilot.py) per-tile operations at "
                       f"N={a.n}, b={a.b}: 4 x (24 tile compressions, 1 POTRF, 32 panel solves/diag updates, 96 "
                       f"step-0 recompressions) timed ({wall:.1f} s, setup {setup:.1f} s) and scaled by their counts in "
                       f"one evaluation: {est:.1f} s per log-likelihood; loglik+grad = 7 evaluations (value and "
                       f"central differences in 3 parameters, the reference's only derivative method)")}


def run_reference(a):
    """The reference arm: the reference's algorithm on the host's cores (the oracle, a NumPy/SciPy
    restatement of codes/17_tlr_cholesky_pilot.py with the same LAPACK calls; the reference itself
    is not present where this runs), every BLAS thread the host has.  The K timed steps are K
    consecutive slices of ONE complete evaluation at the workload's size (oracle/cpu_sample.py:
    timed_full_evaluation), so ms_per_step x K is the measured time of one log-likelihood;
    loglik+grad = 7 evaluations (the value and central differences in 3 parameters, the
    reference's only derivative method).  Warm-up: W complete evaluations at N = 4,000, b = 250."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np  # noqa: F401

    from adaptive_tlr_pilots_b200 import synth
    from oracle import tlr_oracle as O
    from oracle.cpu_sample import blas_threads, timed_full_evaluation
    S, y, _, _ = synth.simulate_field(a.n, THETA, order_fn=O.morton_order)
    if a.warmup:
        Sw, yw, _, _ = O.simulate_field(4000, THETA)
        for _ in range(a.warmup):
            timed_full_evaluation(Sw, yw, THETA, 250, "adaptive", a.tau, 1)
    r = timed_full_evaluation(S, y, THETA, a.b, "adaptive", a.tau, a.steps)
    k = len(r["step_seconds"])
    value = 1.0 / (7.0 * r["seconds"])
    sample = (f"one complete evaluation of the oracle's tlr_loglik (the reference's algorithm, NumPy/SciPy) at "
              f"N={a.n}, b={a.b}, adaptive tau={a.tau}: {r['seconds']:.1f} s measured, timed as {k} consecutive "
              f"slices of its {r['stages']} stages (compression rows, factorization steps, solve); loglik+grad = 7 "
              f"evaluations (value and central differences in 3 parameters); loglik {r['loglik']}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": a.gpus,
            "steps": k, "warmup": a.warmup, "ms_per_step": 1e3 * r["seconds"] / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded reference protocol)",
            "config": workload(a), "step_seconds": r["step_seconds"], "seconds_per_loglik": r["seconds"],
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": blas_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_chains_mode(a):
    """Lockstep random-walk chains at the workload's size: every iteration is one batched call of
    all chains' (loglik, gradient) through `workspaces` device workspaces (PlanBatch groups).
    Starts: the reference's dispersed multipliers of theta_0 (README.md:582) cycled over the
    chains; seeds 101, 102, ...; the prior box of codes/19_tlr_mcmc_gpu.py:23."""
    import numpy as np
    import torch

    from adaptive_tlr_pilots_b200 import inference as I
    from adaptive_tlr_pilots_b200 import synth
    S, y, _, _ = synth.simulate_field(a.n, THETA, device=0)
    mult = np.array([[1.3, 0.8, 1.5], [0.6, 1.4, 0.5], [2.0, 0.5, 2.0], [0.8, 1.2, 0.8]])
    starts = np.log(np.array(THETA)[None, :] * mult[np.arange(a.chains) % 4])
    obj = I.TLRObjective(S, y, a.b, "adaptive", a.tau, precision=a.precision, batch=a.chains,
                         workspaces=a.workspaces)
    obj.batch(starts[: min(a.chains, a.workspaces)])  # warm-up: one group
    free_b, total_b = torch.cuda.mem_get_info(0)
    torch.cuda.synchronize()
    e0 = obj.evals
    t0 = time.perf_counter()
    out = I.run_chains(obj, starts, iters=a.chain_iters, burn=a.chain_iters, seeds=list(range(101, 101 + a.chains)))
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    evals = obj.evals - e0  # every chain's start, then the proposals inside the prior box
    print(json.dumps({"mode": "chains", "config": dict(workload(a), chains=a.chains, workspaces=a.workspaces,
                                                        iters=a.chain_iters, kind="rw"),
                      "evals": evals, "seconds": dt, "evals_per_s": evals / dt,
                      "acceptance": out["acceptance"], "failures": out["failures"],
                      "device_used_gb": (total_b - free_b) / 1e9, "device_gb": total_b / 1e9}), flush=True)


def run_blockrow_mode(a):
    """One FP64 log-likelihood at the workload's size split over the ranks (blockrow.py: block row i
    on rank i % world, one broadcast and one all-gather per step); every rank evaluates the same
    theta and gets the same value.  Timed on the device, max over ranks; `value` = evaluations per
    second of the whole job (strong scaling: the work per evaluation is fixed)."""
    import torch

    import adaptive_tlr_pilots_b200 as tlr
    from adaptive_tlr_pilots_b200 import blockrow, synth
    from adaptive_tlr_pilots_b200.replicas import Replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    S, y, _, _ = synth.simulate_field(a.n, THETA, device=local)
    torch.cuda.empty_cache()
    plan = tlr.Plan(a.n, a.b, cap=64, device=local)
    plan.set_data(S, y)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(a.warmup):
        ev = blockrow.evaluate_distributed(plan, THETA, "adaptive", a.tau)
    rep.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(a.steps):
        ev = blockrow.evaluate_distributed(plan, THETA, "adaptive", a.tau)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = rep.max_over_ranks(e0.elapsed_time(e1)) / a.steps
    if rep.rank == 0:
        print(json.dumps({"metric": "TLR log-likelihood evals/s, one evaluation over all GPUs (block rows cyclic)",
                          "value": 1e3 / ms, "unit": "evals/s", "n_gpus": rep.world, "steps": a.steps,
                          "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": {**{k: v for k, v in workload(a).items()
                                        if k not in ("theta_per_step", "batch", "forward", "precision")},
                                     "precision": "fp64", "parallelism": f"block-row cyclic x{rep.world}"},
                          "loglik": ev.loglik, "stored_factor": ev.info.get("stored_factor")}), flush=True)
    plan.close()
    rep.close()


def main():
    a = parse()
    if a.blockrow:
        run_blockrow_mode(a)
        return
    if a.chains > 0:
        run_chains_mode(a)
        return
    if a.plain_steps < 0:
        a.plain_steps = a.steps * a.batch  # as many plain evaluations as batched ones
    if a.impl == "reference":
        for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
            os.environ.setdefault(var, str(os.cpu_count() or 1))  # every host thread for the BLAS
        run_reference(a)
        return
    import numpy as np
    import torch

    import adaptive_tlr_pilots_b200 as tlr
    from adaptive_tlr_pilots_b200 import synth

    from adaptive_tlr_pilots_b200.replicas import Replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rep = Replicas("nccl")  # one replica per GPU: independent evaluations, no data-path exchange
    world, rank = rep.world, rep.rank
    barrier, max_over_ranks = rep.barrier, rep.max_over_ranks

    if a.sim == "dense":
        S, y, _, _ = synth.simulate_field(a.n, THETA, device=local)
        sim_info = None
    else:  # N where no dense factor fits: the reference's --sim tlr protocol (17:326-339)
        S, y, _, _, sim_info = synth.simulate_field_tlr(a.n, THETA, b=a.b, device=local)
    # dense FP64 oracle at the bench's theta (cuSOLVER through torch; not part of the timed path)
    dense, gdense = (synth.dense_loglik_grad_gpu(S, y, THETA, device=local) if rank == 0 and a.dense
                     and a.sim == "dense" else (None, None))
    torch.cuda.empty_cache()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # the plain FP64 path (every step in FP64, one theta per evaluation): the comparison leg
    plain = None
    if a.plain_steps > 0:
        plan = tlr.Plan(a.n, a.b, cap=64, device=local)
        plan.set_data(S, y)
        plan.set_precision("fp64")
        plan.set_graphs(bool(a.graphs))
        ev64 = plan.evaluate(THETA, "adaptive", a.tau, grad=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(a.plain_steps):
            ev64 = plan.evaluate(THETA, "adaptive", a.tau, grad=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms64 = max_over_ranks(e0.elapsed_time(e1)) / a.plain_steps
        plain = {"value": world * 1e3 / ms64, "unit": "evals/s", "ms_per_step": ms64, "steps": a.plain_steps,
                 "loglik": ev64.loglik, "grad": ev64.grad.tolist(), "batch": 1, "precision": "fp64"}
        plan.close()
        torch.cuda.empty_cache()

    # the headline: B parameter vectors per step (chains near the mode, the first at theta), each
    # step one batched call through the public PlanBatch / tlr_loglik_grad_batch
    B = a.batch
    rng = np.random.default_rng(20261021)
    thetas = np.array(THETA)[None, :] * np.exp(0.05 * rng.standard_normal((B, 3)))
    thetas[0] = THETA
    pb = tlr.PlanBatch(a.n, a.b, B, cap=64, device=local, precision=a.precision)
    for p in pb.plans:
        p.set_graphs(bool(a.graphs))
    pb.set_data(S, y)
    free_b, total_b = torch.cuda.mem_get_info(local)
    for _ in range(a.warmup):
        out = pb.evaluate(thetas, "adaptive", a.tau)
    for p in pb.plans:
        p.kernel_stats(reset=True)
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(a.steps):
        out = pb.evaluate(thetas, "adaptive", a.tau)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms_max = max_over_ranks(e0.elapsed_time(e1))
    stats = {}
    for p in pb.plans:
        for k, v in p.kernel_stats(reset=True).items():
            acc = stats.setdefault(k, dict(ms=0.0, launches=0, flops=0.0, bytes=0.0))
            for f in acc:
                acc[f] += v[f]
    # the roofline of the dominant kernel, from one evaluation of one plan alone (batch 1, every
    # launch bracketed by two events on its stream), so that no other plan's work lies inside a
    # kernel's event interval: the per-kernel table, the dominant kernel and its mean launch time
    p0 = pb.plans[0]
    p0.set_profiling(True)
    torch.cuda.synchronize()
    t_one = time.perf_counter()
    p0.evaluate(THETA, "adaptive", a.tau, grad=True)
    torch.cuda.synchronize()
    t_one = time.perf_counter() - t_one
    prof_stats = p0.kernel_stats(reset=True)
    p0.set_profiling(False)
    ll0, g0, st0 = out[0]
    info0 = pb.plans[0].evaluate(THETA, "adaptive", a.tau).info  # storage of the factor at theta_0

    # end to end through the public API: every step copies the sites and observations from pinned
    # host memory to the device, evaluates the batch and reads the results back
    S_pin = torch.from_numpy(np.ascontiguousarray(S)).pin_memory()
    y_pin = torch.from_numpy(np.ascontiguousarray(y)).pin_memory()
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(a.steps):
        pb.set_data(S_pin, y_pin)
        out_e2e = pb.evaluate(thetas, "adaptive", a.tau)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1))
    h2d = S_pin.numel() * 8 + y_pin.numel() * 8 + thetas.nbytes
    d2h = B * (8 + 3 * 8 + 4)
    pb.close()

    if rank == 0:
        pk, pk_kind = peaks()
        launches = int(sum(v["launches"] for v in stats.values()))
        top = max(prof_stats, key=lambda k: prof_stats[k]["ms"])
        st = prof_stats[top]
        per_launch_ms = st["ms"] / max(st["launches"], 1)
        achieved_gbs = st["bytes"] / max(st["launches"], 1) / (per_launch_ms * 1e-3) / 1e9
        roof = {"kernel": top, "bound": "hbm", "achieved": achieved_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved_gbs / pk["hbm_gbs"], "peak_kind": pk_kind,
                # DRAM bytes per launch from one ncu capture of this kernel on this workload
                "traffic": (RC_TRAFFIC_N50K if top == "recompress" and (a.n, a.b, a.tau) == (50000, 500, 0.9)
                            else None),
                "traffic_source": RC_TRAFFIC_SOURCE,
                "algorithmic_bytes_per_launch": st["bytes"] / max(st["launches"], 1),
                "fp64_tflops": st["flops"] / max(st["launches"], 1) / (per_launch_ms * 1e-3) / 1e12,
                "fp64_peak_nominal_tflops": 37.0,
                "timing": "one evaluation of one plan alone (batch 1), every launch between two CUDA events on "
                          "its stream; achieved = the kernel's own algorithmic bytes per launch / mean launch time",
                "share": st["ms"] / sum(v["ms"] for v in prof_stats.values()),
                "per_launch_ms": per_launch_ms, "launches_per_eval": st["launches"],
                "kernel_ms_per_eval": st["ms"], "eval_wall_ms": 1e3 * t_one}
        # per-kernel table of the profiled evaluation (one plan alone: kernels on its side stream,
        # POTRF and the alpha solve, overlap those of the main stream, so the column does not add
        # up to the evaluation's wall time)
        kern = {k: {"ms_per_eval": v["ms"], "launches_per_eval": v["launches"],
                    "gflop_per_eval": v["flops"] / 1e9, "gb_per_eval": v["bytes"] / 1e9}
                for k, v in prof_stats.items() if v["launches"]}
        value = world * a.steps * B / (ms_max / 1e3)
        line = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f64+tf32x3",
                "data": ("synthetic (seeded reference protocol, y = L z with the dense FP64 Cholesky)" if a.sim == "dense"
                         else "synthetic (seeded reference protocol, y = L z with a tight TLR factor: no dense factor fits)"),
                "config": dict(workload(a), parallelism=f"replicas x{world}"),
                "loglik": ll0, "dense_loglik": dense,
                "abs_dloglik_vs_dense": None if (dense is None or ll0 is None) else abs(ll0 - dense),
                "grad": None if g0 is None else g0.tolist(), "dense_grad": None if gdense is None else list(gdense),
                "grad_rel_err_vs_dense": None if (gdense is None or g0 is None) else
                float(np.linalg.norm(g0 - gdense) / np.linalg.norm(gdense)),
                "plain_fp64": plain,
                "speedup_vs_plain_fp64": None if plain is None else value / plain["value"],
                "abs_dloglik_vs_plain_fp64": None if (plain is None or ll0 is None) else abs(ll0 - plain["loglik"]),
                "grad_rel_err_vs_plain_fp64": None if (plain is None or g0 is None) else
                float(np.linalg.norm(g0 - np.array(plain["grad"])) / np.linalg.norm(plain["grad"])),
                "e2e": {"value": world * a.steps * B / (ms_e2e / 1e3), "unit": "evals/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "gpu_launches": launches, "roofline": roof, "kernels": kern, "clocks": clocks,
                "memory": {"device_used_gb_with_batch": (total_b - free_b) / 1e9, "device_gb": total_b / 1e9,
                           "per_plan_gb_approx": (total_b - free_b) / 1e9 / B},
                "storage": {"stored_factor": info0.get("stored_factor"),
                            "fraction_of_dense_factor": None if info0.get("stored_factor") is None else
                            info0["stored_factor"] / (a.n * (a.n + 1) / 2),
                            "mean_rank_factor": info0.get("mean_rank_factor"),
                            "max_rank_factor": info0.get("max_rank_factor")},
                "simulation": sim_info}
        if world == 1 and a.cpu_sample:
            line["cpu_baseline"] = cpu_baseline(S, y, a)
        print(json.dumps(line), flush=True)
    tlr.release_plans()
    rep.close()


if __name__ == "__main__":
    main()
