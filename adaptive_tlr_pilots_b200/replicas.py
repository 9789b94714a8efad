"""One process per GPU for independent evaluations (parameter vectors, chains).

The log-likelihood path has no exchange between evaluations: N GPUs run N replicas, each on its
own share of the parameter vectors or chains, and only the bookkeeping crosses processes: a
barrier around timed regions, the maximum of the ranks' device times, and the gathering of
results on rank 0.  The reference runs one evaluation or chain per process and has no
multi-GPU path (codes/19_tlr_mcmc_gpu.py:170-202 runs its chains one after another).

Launch as `python -m torch.distributed.run --nproc-per-node N ...`; RANK, LOCAL_RANK,
WORLD_SIZE, MASTER_ADDR and MASTER_PORT come from the environment.  With WORLD_SIZE unset or 1
nothing is initialised and every call is local.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    """Process-group plumbing for replicas; backend 'nccl' on GPUs (default when CUDA is
    available), 'gloo' on CPU.  `timeout_s` bounds every collective, so ranks waiting for a rank
    that died or never joined end with an error instead of waiting for good."""

    def __init__(self, backend: str | None = None, timeout_s: float = 600.0):
        import torch
        import torch.distributed as dist

        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        self._dist = dist
        self._torch = torch
        if self.world > 1:
            kw = {}
            if self.backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(self.backend, timeout=timedelta(seconds=timeout_s), **kw)

    def _device(self):
        return self._torch.device("cuda", self.local) if self.backend == "nccl" else self._torch.device("cpu")

    def barrier(self) -> None:
        if self.world > 1:
            self._dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """The largest of the ranks' values (device times of a timed region are combined this way)."""
        t = self._torch.tensor([float(x)], dtype=self._torch.float64, device=self._device())
        if self.world > 1:
            self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def shard(self, n_items: int) -> range:
        """This rank's contiguous share of n_items independent items (sizes differ by at most one)."""
        base, extra = divmod(n_items, self.world)
        start = self.rank * base + min(self.rank, extra)
        return range(start, start + base + (1 if self.rank < extra else 0))

    def gather(self, local: list) -> list | None:
        """Every rank's list, concatenated in rank order, on rank 0 (None elsewhere)."""
        if self.world == 1:
            return list(local)
        parts = [None] * self.world if self.rank == 0 else None
        self._dist.gather_object(list(local), parts, dst=0)
        if self.rank != 0:
            return None
        return [x for p in parts for x in p]

    def rate(self, units_per_rank: float, ms: float) -> float:
        """Whole-job throughput: every rank processed units_per_rank in at most ms milliseconds."""
        return self.world * units_per_rank / (ms / 1e3)

    def close(self) -> None:
        if self.world > 1 and self._dist.is_initialized():
            self._dist.destroy_process_group()
