"""The block-row cyclic schedule (adaptive_tlr_pilots_b200/blockrow.py) on the CPU: two gloo
processes, and three lockstep ranks in one process.

The ranks' device calls are replaced by `DenseSteps`, a test double that follows the same buffer
protocol with dense tiles (the reference's own multi-GPU tile Cholesky, codes/13_multigpu_tile_
cholesky.py:45-79, with numpy on the CPU): the broadcast carries L_kk and z_k, the all-gather the
panel tiles L_ik of every rank in rank order, the sum the log-determinant and quadratic-form parts.
The log-determinant and quadratic form must equal a dense Cholesky's, so every exchange has to
reach the right ranks in the right order."""
import json
import os
import socket
import sys

import numpy as np
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N, B = 60, 8


def _problem():
    rng = np.random.default_rng(7)
    S = rng.random((N, 2))
    d = np.sqrt(((S[:, None, :] - S[None, :, :]) ** 2).sum(-1))
    x = np.sqrt(3.0) * d / 0.3
    K = (1.0 + x) * np.exp(-x) + 0.05 * np.eye(N)
    return K, rng.standard_normal(N)


class DenseSteps:
    """One rank of a dense block-row cyclic tile Cholesky, speaking blockrow's protocol."""

    def __init__(self, K, y, b, rank, world):
        self.rank, self.world, self.b = rank, world, b
        self.bounds = [(s, min(s + b, len(y))) for s in range(0, len(y), b)]
        self.nB = len(self.bounds)
        self.own = [i for i in range(self.nB) if i % world == rank]
        blk = lambda i, j: K[self.bounds[i][0]:self.bounds[i][1], self.bounds[j][0]:self.bounds[j][1]].copy()
        self.A = {(i, j): blk(i, j) for i in self.own for j in range(i + 1)}
        self.rhs = {i: y[self.bounds[i][0]:self.bounds[i][1]].copy() for i in self.own}
        self.L, self.z, self.col = {}, {}, {}
        self.ld, self.q = np.zeros(self.nB), np.zeros(self.nB)
        self.diag = torch.zeros(b * b + b, dtype=torch.float64)
        self.panel = torch.zeros(self.panel_len(0), dtype=torch.float64)
        self.gathered = torch.zeros(self.panel_len(0) * world, dtype=torch.float64)
        self.sums = torch.zeros(2 * self.nB, dtype=torch.float64)

    def owner(self, k):
        return k % self.world

    def _rows(self, k, src):
        return [i for i in range(k + 1, self.nB) if i % self.world == src]

    def panel_len(self, k):
        most = max(len(self._rows(k, w)) for w in range(self.world))
        return 8 + most * self.b * self.b

    def _factor(self, k):
        L = np.linalg.cholesky(self.A[(k, k)])
        self.L[k] = L
        self.z[k] = np.linalg.solve(L, self.rhs[k])
        self.ld[k] = 2.0 * np.log(np.diag(L)).sum()
        self.q[k] = self.z[k] @ self.z[k]

    def begin(self, theta, rule, value):
        if self.owner(0) == self.rank:
            self._factor(0)

    def pack_diag(self, k):
        m = self.L[k].shape[0]
        self.diag.zero_()
        self.diag[: m * m] = torch.from_numpy(self.L[k].ravel())
        self.diag[self.b * self.b: self.b * self.b + m] = torch.from_numpy(self.z[k])

    def unpack_diag(self, k):
        if self.owner(k) == self.rank:
            return
        m = self.bounds[k][1] - self.bounds[k][0]
        d = self.diag.numpy()
        self.L[k] = d[: m * m].reshape(m, m).copy()
        self.z[k] = d[self.b * self.b: self.b * self.b + m].copy()

    def solve(self, k):
        for i in self._rows(k, self.rank):
            Lik = np.linalg.solve(self.L[k], self.A[(i, k)].T).T
            self.col[(i, k)] = Lik
            self.rhs[i] -= Lik @ self.z[k]

    def pack_panel(self, k):
        self.panel.zero_()
        for q, i in enumerate(self._rows(k, self.rank)):
            t = self.col[(i, k)]
            off = 8 + q * self.b * self.b
            self.panel[off: off + t.size] = torch.from_numpy(t.ravel())

    def unpack_panel(self, k):
        n = self.panel_len(k)
        g = self.gathered.numpy()
        for src in range(self.world):
            for q, j in enumerate(self._rows(k, src)):
                shape = (self.bounds[j][1] - self.bounds[j][0], self.bounds[k][1] - self.bounds[k][0])
                off = src * n + 8 + q * self.b * self.b
                self.col[(j, k)] = g[off: off + shape[0] * shape[1]].reshape(shape).copy()

    def update(self, k):
        for i in self._rows(k, self.rank):
            for j in range(k + 1, i + 1):
                self.A[(i, j)] -= self.col[(i, k)] @ self.col[(j, k)].T
        if k + 1 < self.nB and self.owner(k + 1) == self.rank:
            self._factor(k + 1)

    def pack_sums(self):
        mine = np.array([k % self.world == self.rank for k in range(self.nB)], dtype=float)
        self.sums[:] = torch.from_numpy(np.concatenate([self.ld * mine, self.q * mine]))

    def finish(self):
        s = self.sums.numpy()
        return float(s[: self.nB].sum()), float(s[self.nB:].sum())


def _dense():
    K, y = _problem()
    L = np.linalg.cholesky(K)
    z = np.linalg.solve(L, y)
    return 2.0 * np.log(np.diag(L)).sum(), z @ z


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    from adaptive_tlr_pilots_b200 import blockrow
    from test_blockrow_gloo import DenseSteps, _problem
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    K, y = _problem()
    steps = DenseSteps(K, y, B, rank, world)
    logdet, quad = blockrow.run_rank(blockrow.rank_steps(steps, None, None, None), blockrow.TorchExchange())
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(dict(logdet=logdet, quad=quad), f)


def test_two_ranks_on_gloo(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    ld, q = _dense()
    for r in range(world):
        got = json.load(open(tmp_path / f"rank{r}.json"))
        assert abs(got["logdet"] - ld) <= 1e-11 * abs(ld), (got, ld)
        assert abs(got["quad"] - q) <= 1e-11 * abs(q), (got, q)


def test_lockstep_ranks_in_one_process():
    from adaptive_tlr_pilots_b200 import blockrow
    K, y = _problem()
    ld, q = _dense()
    for world in (1, 3, 8):  # 8 ranks: every rank owns exactly one block row
        steps = [DenseSteps(K, y, B, r, world) for r in range(world)]
        out = blockrow.run_lockstep([blockrow.rank_steps(s, None, None, None) for s in steps])
        for got_ld, got_q in out:
            assert abs(got_ld - ld) <= 1e-11 * abs(ld) and abs(got_q - q) <= 1e-11 * abs(q)
