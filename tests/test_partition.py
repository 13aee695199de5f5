"""The row-partitioned PageRank's loop (pg_warren_b200/partition.py) on two
gloo ranks (CPU): each rank iterates its rows, the ranks sum the parts' L1
changes and dangling ranks and gather each other's rows of the messages,
and every rank ends with the unsharded solve's ranks and iteration count
(the oracle's, compute/pagerank/mod.rs:96-151).  The parts here are a host
implementation of the same methods the GPU parts (wc_pagerank_part_*)
have; the loop, the exchange and the stop test are the library's."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from pg_warren_b200.partition import solve

N = 300


def graph():
    """A random graph with dangling nodes (0..9 have no out-edges)."""
    rng = np.random.default_rng(21)
    pairs = {(int(a), int(b)) for a, b in rng.integers(0, N, (2400, 2)) if a != b and a >= 10}
    rows = [[] for _ in range(N)]
    for a, b in sorted(pairs):
        rows[a].append(b)
    offsets = np.zeros(N + 1, np.uint64)
    offsets[1:] = np.cumsum([len(r) for r in rows])
    targets = np.array([t for r in rows for t in r], np.uint32)
    return offsets, targets


class HostParts:
    """The parts' methods on the host, in dense-id order: the reference's
    arithmetic per row (the pull folded in ascending source order, advance,
    spread)."""

    def __init__(self, offsets, targets, damping, tol, max_iter):
        self.n = len(offsets) - 1
        self.out = np.diff(offsets).astype(np.float64)
        self.rev = [[] for _ in range(self.n)]
        for s in range(self.n):
            for e in range(int(offsets[s]), int(offsets[s + 1])):
                self.rev[int(targets[e])].append(s)
        self.damping, self.tol, self.max_iter = damping, tol, max_iter
        self.ranks2 = torch.zeros((2, self.n), dtype=torch.float64)
        self.messages2 = torch.zeros((2, self.n), dtype=torch.float64)

    def rows(self, parts):
        entries = np.cumsum([0] + [len(r) for r in self.rev])
        bounds = [0]
        for p in range(1, parts):
            bounds.append(int(np.searchsorted(entries, entries[-1] * p / parts)))
        return np.array(bounds + [self.n])

    def begin(self, parts, part):
        class Info:
            pass
        b = self.rows(parts)
        self.lo, self.hi = int(b[part]), int(b[part + 1])
        self.start = 1.0 / self.n
        self.teleport = 1.0 - self.damping
        x, m = self.ranks2[0].numpy(), self.messages2[0].numpy()
        dangling = 0.0
        for i in range(self.n):
            x[i] = self.start
            m[i] = x[i] / self.out[i] if self.out[i] > 0 else 0.0
            if not self.out[i] > 0:
                dangling = dangling + x[i]
        info = Info()
        info.dangling = dangling
        info.threshold = self.n * self.tol if self.tol is not None else 0.0
        return info

    def step(self, it, dangling):
        cur, nxt = it & 1, (it + 1) & 1
        m = self.messages2[cur].numpy()
        xo, xn, mn = self.ranks2[cur].numpy(), self.ranks2[nxt].numpy(), self.messages2[nxt].numpy()
        delta = dangling_out = 0.0
        p = self.start
        for i in range(self.lo, self.hi):
            y = 0.0
            for k, j in enumerate(self.rev[i]):
                y = m[j] if k == 0 else y + m[j]
            nx = self.damping * (y + dangling * p) + self.teleport * p
            delta = delta + abs(nx - xo[i])
            xn[i] = nx
            mn[i] = nx / self.out[i] if self.out[i] > 0 else 0.0
            if not self.out[i] > 0:
                dangling_out = dangling_out + nx
        return delta, dangling_out

    def end(self, iterations, out=None):
        return self.ranks2[iterations & 1].numpy().copy()


def _rank(rank, world, port, tol, max_iter, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, tgt = graph()
        parts = HostParts(off, tgt, 0.85, tol, max_iter)
        ranks, its = solve(parts, max_iter, tol is not None, collective_device="cpu")
        np.save(out + f"_{rank}.npy", ranks)
        np.save(out + f"_{rank}_its.npy", np.array([its, parts.lo, parts.hi]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("tol,max_iter", [(1e-10, 100), (None, 7)])
def test_two_gloo_ranks_equal_the_unpartitioned_solve(tmp_path, tol, max_iter):
    out = str(tmp_path / "pr")
    mp.start_processes(_rank, args=(2, _free_port(), tol, max_iter, out), nprocs=2,
                       start_method="spawn")
    off, tgt = graph()
    og = O.Graph.from_csr(N, off, tgt)
    want, want_its, _, _ = O.pagerank(og, 0.85, tol, max_iter)
    spans = []
    for rank in range(2):
        got = np.load(out + f"_{rank}.npy")
        its, lo, hi = np.load(out + f"_{rank}_its.npy")
        spans.append((lo, hi))
        assert its == want_its
        assert np.abs(got - want).sum() / want.sum() <= 1e-12
    assert spans[0][0] == 0 and spans[0][1] == spans[1][0] and spans[1][1] == N


def test_without_a_process_group_one_part_runs_every_row():
    off, tgt = graph()
    parts = HostParts(off, tgt, 0.85, 1e-10, 100)
    ranks, its = solve(parts, 100, True)
    og = O.Graph.from_csr(N, off, tgt)
    want, want_its, _, _ = O.pagerank(og, 0.85, 1e-10, 100)
    assert its == want_its and np.abs(ranks - want).sum() / want.sum() <= 1e-12
