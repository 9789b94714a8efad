"""Block-row cyclic TLR factorization over several ranks (codes/13_multigpu_tile_cholesky.py:45-79,
tile_cholesky_multi, with the TLR tiles and rank rule of codes/17_tlr_cholesky_pilot.py:137-215).

Block row i lives on rank i % world (13:45-50).  At step k the owner of row k forms and factors the
diagonal tile and every rank receives it (13:52-66: one broadcast of L_kk and of the forward-solve
block z_k); every rank solves its own panel tiles (i, k) and all ranks exchange them (one
all-gather: the trailing update of row i needs the panel tiles of every row j < i); every rank then
recompresses the trailing pairs (i, j) of its own rows (13:68-76), and the owner of row k + 1 forms
and factors the next diagonal tile beside that.  The log-determinant and quadratic-form parts and
the initial ranks are summed at the end.

The device work is the library's (include/tlr_b200.h, tlr_dist_*); this module only runs the
steps and moves the three exchange buffers:

* `evaluate_distributed(plan, ...)`: one process per GPU, buffers moved by torch.distributed
  (NCCL over NVLink: broadcast, all_gather_into_tensor, all_reduce), every rank in the same order;
* `evaluate_lockstep(plans, ...)`: `world` partitioned plans in one process (one GPU), buffers moved
  by device copies, the ranks' steps interleaved; the factorization is the same, tile for tile.

Both run `rank_steps`, a generator that issues one rank's library calls and yields each exchange
as a request, so the order of the steps is written once.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .tlr import RULES, Evaluation, Plan, _torch


class RankSteps:
    """The library calls of one rank of a partitioned plan (tlr_dist_*), with its exchange buffers
    as float64 device tensors."""

    def __init__(self, plan: Plan, rank: int, world: int):
        torch = _torch()
        self.plan, self.rank, self.world = plan, int(rank), int(world)
        plan.set_partition(rank, world)
        lib, h = plan.lib, plan.handle
        self.nB = plan.nB
        n_diag = int(lib.tlr_dist_buffer_doubles(h, _lib.DIST_DIAG, 0))
        n_panel = int(lib.tlr_dist_buffer_doubles(h, _lib.DIST_PANEL, -1))
        n_sums = int(lib.tlr_dist_buffer_doubles(h, _lib.DIST_SUMS, 0))
        kw = dict(dtype=torch.float64, device=plan.dev)
        with torch.cuda.stream(plan.stream):  # filled on the stream the library then writes them on
            self.diag = torch.zeros(n_diag, **kw)
            self.panel = torch.zeros(n_panel, **kw)
            self.gathered = torch.zeros(n_panel * self.world, **kw)
            self.sums = torch.zeros(n_sums, **kw)

    def owner(self, k: int) -> int:
        return k % self.world

    def panel_len(self, k: int) -> int:
        return int(self.plan.lib.tlr_dist_buffer_doubles(self.plan.handle, _lib.DIST_PANEL, k))

    def _call(self, name, *args):
        _lib.check(getattr(self.plan.lib, name)(self.plan.handle, *args))

    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    def begin(self, theta, rule, value):
        th = (ctypes.c_double * 3)(*[float(v) for v in theta])
        self.plan._apply_kernel()
        self._call("tlr_dist_begin", th, RULES[rule], float(value))

    def pack_diag(self, k):
        self._call("tlr_dist_pack_diag", k, self._ptr(self.diag))

    def unpack_diag(self, k):
        self._call("tlr_dist_unpack_diag", k, self._ptr(self.diag))

    def solve(self, k):
        self._call("tlr_dist_solve_step", k)

    def pack_panel(self, k):
        self._call("tlr_dist_pack_panel", k, self._ptr(self.panel))

    def unpack_panel(self, k):
        self._call("tlr_dist_unpack_panel", k, self._ptr(self.gathered))

    def update(self, k):
        self._call("tlr_dist_update_step", k)

    def pack_sums(self):
        self._call("tlr_dist_pack_sums", self._ptr(self.sums))

    def finish(self) -> Evaluation:
        p = self.plan
        ll = ctypes.c_double(0.0)
        info = _lib.TlrInfo()
        fr = np.zeros(max(p.ntiles, 1), dtype=np.int32)
        sr = np.zeros(max(p.ntiles, 1), dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        rc = _lib.check(p.lib.tlr_dist_finish(p.handle, self._ptr(self.sums), ctypes.byref(ll), ctypes.byref(info),
                                              fr.ctypes.data_as(ip), sr.ctypes.data_as(ip)))
        d = dict(completed=bool(info.completed), stored_sigma=int(info.stored_sigma),
                 max_rank_sigma=int(info.max_rank_sigma), rank=self.rank, world=self.world)
        if rc == 0:
            d.update(stored_factor=int(info.stored_factor), mean_rank_factor=float(info.mean_rank_factor),
                     max_rank_factor=int(info.max_rank_factor), logdet=float(info.logdet), quad=float(info.quad))
        else:
            d.update(failed_at=int(info.failed_at))
        return Evaluation(rc, float(ll.value) if rc == 0 else None, d, fr[: p.ntiles], sr[: p.ntiles], None)


def rank_steps(steps: RankSteps, theta, rule, value):
    """One rank's factorization and log-likelihood.  Yields each exchange as a request:
    ("bcast", tensor, src) — every rank's tensor takes the src rank's; ("gather", out, inp) — out
    takes every rank's inp in rank order; ("sum", tensor) — every rank's tensor takes the sum.
    Returns the rank's Evaluation (the same on every rank)."""
    steps.begin(theta, rule, value)
    for k in range(steps.nB):
        if steps.owner(k) == steps.rank:
            steps.pack_diag(k)
        yield ("bcast", steps.diag, steps.owner(k))
        steps.unpack_diag(k)  # the owner keeps its own
        steps.solve(k)
        m = steps.panel_len(k)
        steps.pack_panel(k)
        yield ("gather", steps.gathered[: m * steps.world], steps.panel[:m])
        steps.unpack_panel(k)
        steps.update(k)
    steps.pack_sums()
    yield ("sum", steps.sums)
    return steps.finish()


class TorchExchange:
    """The exchanges over a torch.distributed process group (NCCL between GPUs; gloo moves CPU
    tensors).  Ranks are the group's; without an initialised process group, one local rank."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.local = not dist.is_initialized()  # no process group: one rank, every exchange local
        self.rank = 0 if self.local else dist.get_rank(group)
        self.world = 1 if self.local else dist.get_world_size(group)
        self._into = not self.local and dist.get_backend(group) == "nccl"

    def _global(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def serve(self, req):
        kind = req[0]
        if self.local:
            if kind == "gather":
                req[1].copy_(req[2])
            return
        if kind == "bcast":
            self.dist.broadcast(req[1], src=self._global(req[2]), group=self.group)
        elif kind == "gather":
            out, inp = req[1], req[2]
            if self._into:
                self.dist.all_gather_into_tensor(out, inp, group=self.group)
            else:
                parts = list(out.view(self.world, -1).unbind(0))
                self.dist.all_gather(parts, inp, group=self.group)
        elif kind == "sum":
            self.dist.all_reduce(req[1], group=self.group)
        else:
            raise ValueError(f"unknown exchange {kind!r}")


def run_rank(gen, exchange):
    """Drive one rank's generator, serving its requests with `exchange`; returns its result."""
    try:
        req = next(gen)
        while True:
            exchange.serve(req)
            req = gen.send(None)
    except StopIteration as stop:
        return stop.value


def run_lockstep(gens, sync=False):
    """Drive the generators of all ranks in one process: each exchange is served by copies once
    every rank has issued it (on the current stream; with sync, between two device-wide
    synchronisations, for ranks on different streams).  Returns the ranks' results."""
    world = len(gens)
    reqs = [next(g) for g in gens]
    while True:
        kinds = {r[0] for r in reqs}
        if len(kinds) != 1:
            raise RuntimeError(f"ranks out of step: {sorted(kinds)}")
        fence = sync and reqs[0][1].device.type == "cuda"
        if fence:
            _torch().cuda.synchronize()
        kind = reqs[0][0]
        if kind == "bcast":
            src = reqs[0][2]
            for r in range(world):
                if r != src:
                    reqs[r][1].copy_(reqs[src][1])
        elif kind == "gather":
            parts = [r[2] for r in reqs]
            for r in reqs:
                for w, part in enumerate(parts):
                    r[1][w * part.numel():(w + 1) * part.numel()].copy_(part)
        elif kind == "sum":
            total = reqs[0][1].clone()
            for r in reqs[1:]:
                total += r[1]
            for r in reqs:
                r[1].copy_(total)
        if fence:
            _torch().cuda.synchronize()
        results, nxt, done = [None] * world, [None] * world, 0
        for w, g in enumerate(gens):
            try:
                nxt[w] = g.send(None)
            except StopIteration as stop:
                results[w] = stop.value
                done += 1
        if done == world:
            return results
        if done:
            raise RuntimeError("ranks out of step: some finished early")
        reqs = nxt


def evaluate_distributed(plan: Plan, theta, rule, value, group=None) -> Evaluation:
    """The TLR log-likelihood of `plan`'s data over the ranks of a torch.distributed group, block
    rows cyclic over the ranks.  Every rank calls this with its own plan (same n, b, data, theta)
    and receives the same Evaluation.  A tile rank above the capacity grows every rank's plan (the
    failure reaches all ranks) and the evaluation is repeated.  Any other error raises on the rank
    that met it; the other ranks then wait in their next collective until the process group's
    timeout ends it (create the group with a short timeout)."""
    ex = TorchExchange(group)
    while True:
        steps = _steps_for(plan, ex.rank, ex.world)
        try:
            # the collectives are ordered on the plan's stream (torch's NCCL calls wait for the
            # current stream and make it wait for them)
            with _torch().cuda.stream(plan.stream):
                return run_rank(rank_steps(steps, theta, rule, value), ex)
        except _lib.TlrError as e:
            if e.code != _lib.ERR_RANK_CAP or not plan.grow():
                raise


def evaluate_lockstep(plans, theta, rule, value):
    """The same factorization with len(plans) ranks in one process (every plan partitioned as one
    rank): the ranks' steps interleaved, the exchanges device copies.  Returns the ranks' results."""
    torch = _torch()
    world = len(plans)
    shared = len({p.stream for p in plans}) == 1
    while True:
        steps = [_steps_for(p, r, world) for r, p in enumerate(plans)]
        try:
            if shared:  # one stream orders the plans' launches and the copies between them
                with torch.cuda.stream(plans[0].stream):
                    return run_lockstep([rank_steps(s, theta, rule, value) for s in steps])
            return run_lockstep([rank_steps(s, theta, rule, value) for s in steps], sync=True)
        except _lib.TlrError as e:
            if e.code != _lib.ERR_RANK_CAP or not all(p.grow() for p in plans):
                raise


def _steps_for(plan: Plan, rank: int, world: int) -> RankSteps:
    s = getattr(plan, "_rank_steps", None)
    if s is None or s.rank != rank or s.world != world or s.plan_cap != plan.cap or s.handle != plan.handle.value:
        s = RankSteps(plan, rank, world)
        s.plan_cap, s.handle = plan.cap, plan.handle.value
        plan._rank_steps = s
    return s
