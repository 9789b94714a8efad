"""Replica plumbing for N GPUs, exercised as two gloo processes on the CPU.

Independent evaluations shard across ranks with no data-path exchange; only the barrier, the
maximum of the ranks' times and the gathering of results cross processes."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from adaptive_tlr_pilots_b200.replicas import Replicas

    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    mx = rep.max_over_ranks(10.0 + rank)           # device times: the job takes as long as its slowest rank
    sh = rep.shard(11)                              # 11 parameter vectors over the ranks
    got = rep.gather([i * i for i in sh])           # each rank evaluates its share; rank 0 collects
    rate = rep.rate(4, mx)
    rep.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(dict(max=mx, shard=[sh.start, sh.stop], gathered=got, rate=rate), f)


def test_two_replicas_on_gloo(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    r = [json.load(open(tmp_path / f"rank{q}.json")) for q in range(world)]
    assert r[0]["max"] == r[1]["max"] == 11.0
    assert r[0]["shard"] == [0, 6] and r[1]["shard"] == [6, 11]   # sizes differ by at most one, no gaps
    assert r[0]["gathered"] == [i * i for i in range(11)]           # rank order, every item once
    assert r[1]["gathered"] is None
    assert r[0]["rate"] == pytest.approx(2 * 4 / 0.011)


def test_single_process_is_local():
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from adaptive_tlr_pilots_b200.replicas import Replicas\n"
            "r = Replicas('gloo'); assert r.world == 1 and list(r.shard(3)) == [0, 1, 2]\n"
            "assert r.max_over_ranks(2.5) == 2.5 and r.gather([1, 2]) == [1, 2]; r.close(); print('ok')" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 runs the reference arm; the others exit 0 without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         env=env, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0 and out.stdout.strip() == "", (out.stdout, out.stderr)


def test_rank_that_never_joins_ends_the_others_with_an_error():
    """Rank 1 of 2 never starts: rank 0's rendezvous ends with an error after its short timeout
    instead of waiting for good (failure made on the host; no GPU involved)."""
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), WORLD_SIZE="2", RANK="0",
               LOCAL_RANK="0")
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from adaptive_tlr_pilots_b200.replicas import Replicas\n"
            "Replicas('gloo', timeout_s=5)\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=240)
    assert out.returncode != 0
