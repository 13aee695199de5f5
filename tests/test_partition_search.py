"""The row-partitioned level search's and product's loops
(pg_warren_b200/partition.py: `search`, `spmv_iterate`) on two and three
gloo ranks (CPU).  Each rank reaches (or multiplies) its own rows; the ranks
sum the next frontier's nodes and out-edges and gather each other's words of
the frontier bitmap (or rows of y), and every rank ends with the unsharded
result: the oracle's level search (traversal/level.rs, bfs.rs:34-45) depths
and its product (compute/product/mod.rs:77-92) iterated.  The parts here are
host implementations of the methods the GPU parts (wc_bfs_part_*,
wc_spmv_part) have; the loops and the exchanges are the library's."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from pg_warren_b200.partition import search, spmv_iterate

N = 700
UNREACHED = 0xFFFFFFFF
DIRS = {"out": 0, "in": 1, "both": 2}


def graph(seed=23):
    """A sparse random graph: several components, rows of every length."""
    rng = np.random.default_rng(seed)
    pairs = {(int(a), int(b)) for a, b in rng.integers(0, N, (1500, 2)) if a != b}
    rows = [[] for _ in range(N)]
    for a, b in sorted(pairs):
        rows[a].append(b)
    offsets = np.zeros(N + 1, np.uint64)
    offsets[1:] = np.cumsum([len(r) for r in rows])
    targets = np.array([t for r in rows for t in r], np.uint32)
    return offsets, targets


class HostBfsParts:
    """The search parts' methods on the host: the part's unvisited rows are
    reached when any neighbour (in the search direction) is in the frontier."""

    def __init__(self, offsets, targets, starts, direction, max_depth):
        self.n = len(offsets) - 1
        fwd = [[int(t) for t in targets[offsets[s]:offsets[s + 1]]] for s in range(self.n)]
        rev = [[] for _ in range(self.n)]
        for s in range(self.n):
            for t in fwd[s]:
                rev[t].append(s)
        self.into = {"out": rev, "in": fwd,
                     "both": [a + b for a, b in zip(rev, fwd)]}[direction]
        self.outof = {"out": fwd, "in": rev,
                      "both": [a + b for a, b in zip(fwd, rev)]}[direction]
        self.starts = [int(s) for s in starts]
        self.max_depth = max_depth
        self.words = (self.n + 63) // 64
        self.frontier2 = torch.zeros(2 * self.words, dtype=torch.int64)
        self.depth = torch.full((self.n,), -1, dtype=torch.int32)

    def frontier(self, level):
        h = (level & 1) * self.words
        return self.frontier2[h: h + self.words]

    def _bits(self, level):
        return self.frontier(level).numpy().view(np.uint64)

    def rows(self, parts):
        work = np.cumsum([0] + [len(r) + 1 for r in self.into])
        bounds = [0]
        for p in range(1, parts):
            r = int(np.searchsorted(work, work[-1] * p / parts))
            bounds.append(max(min((r + 63) // 64 * 64, self.n), bounds[-1]))
        return np.array(bounds + [self.n])

    def begin(self, parts, part):
        class Info:
            pass
        b = self.rows(parts)
        self.lo, self.hi = int(b[part]), int(b[part + 1])
        f = self._bits(0)
        d = self.depth.numpy()
        for s in self.starts:
            f[s // 64] |= np.uint64(1) << np.uint64(s % 64)
            if self.lo <= s < self.hi:
                d[s] = 0
        info = Info()
        nodes = [i for i in range(self.n) if (int(f[i // 64]) >> (i % 64)) & 1]
        info.frontier = len(nodes)
        info.frontier_edges = sum(len(self.outof[u]) for u in nodes)
        return info

    def step(self, level, frontier_edges):
        assert level < (self.max_depth if self.max_depth is not None else 2**32)
        f, nxt = self._bits(level), self._bits(level + 1)
        d = self.depth.numpy()
        lo_w, hi_w = self.lo // 64, (self.hi + 63) // 64
        nxt[lo_w:hi_w] = 0
        count = edges = 0
        for v in range(self.lo, self.hi):
            if d[v] != -1:
                continue
            if any((int(f[u // 64]) >> (u % 64)) & 1 for u in self.into[v]):
                nxt[v // 64] |= np.uint64(1) << np.uint64(v % 64)
                d[v] = level + 1
                count += 1
                edges += len(self.outof[v])
        return count, edges

    def end(self):
        return self.depth


class HostSpmvParts:
    """The product parts' method on the host: the oracle's whole product,
    of which only the part's rows are kept."""

    def __init__(self, offsets, targets, semiring, transpose):
        self.og = O.Graph.from_csr(len(offsets) - 1, offsets, targets)
        self.semiring, self.transpose = semiring, transpose
        self.n = len(offsets) - 1

    def rows(self, parts):
        return np.array([self.n * p // parts for p in range(parts)] + [self.n])

    def apply(self, parts, part, x, y):
        b = self.rows(parts)
        full = y.numpy().copy()
        assert O.product(self.og, self.semiring, x.numpy(), full, transpose=self.transpose) == 0
        y[b[part]:b[part + 1]] = torch.from_numpy(full[b[part]:b[part + 1]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _search_rank(rank, world, port, starts, direction, max_depth, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, tgt = graph()
        parts = HostBfsParts(off, tgt, starts, direction, max_depth)
        depth, levels = search(parts, max_depth)
        np.save(out + f"_{rank}.npy", depth.numpy().view(np.uint32))
        np.save(out + f"_{rank}_span.npy", np.array([parts.lo, parts.hi, levels]))
    finally:
        dist.destroy_process_group()


def expected_depths(starts, direction, max_depth):
    off, tgt = graph()
    og = O.Graph.from_csr(N, off, tgt)
    visits, _ = O.bfs(og, starts, DIRS[direction], max_depth)
    want = np.full(N, UNREACHED, np.uint32)
    for node, depth, _ in visits:
        want[node] = depth
    return want


@pytest.mark.parametrize("world,direction,max_depth",
                         [(2, "out", None), (2, "in", 3), (3, "both", None), (3, "out", 1)])
def test_gloo_ranks_equal_the_unpartitioned_search(tmp_path, world, direction, max_depth):
    starts = [5, 300, 5, 699]
    out = str(tmp_path / "bfs")
    mp.start_processes(_search_rank, args=(world, _free_port(), starts, direction, max_depth, out),
                       nprocs=world, start_method="spawn")
    want = expected_depths(starts, direction, max_depth)
    spans = []
    for rank in range(world):
        got = np.load(out + f"_{rank}.npy")
        lo, hi, levels = np.load(out + f"_{rank}_span.npy")
        spans.append((lo, hi))
        assert np.array_equal(got, want)
        assert lo % 64 == 0
    assert spans[0][0] == 0 and spans[-1][1] == N
    assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))


def test_without_a_process_group_one_part_searches_every_row():
    off, tgt = graph()
    parts = HostBfsParts(off, tgt, [17], "out", None)
    depth, levels = search(parts, None)
    want = expected_depths([17], "out", None)
    assert np.array_equal(depth.numpy().view(np.uint32), want)
    assert levels == int(want[want != UNREACHED].max()) + 1


def _spmv_rank(rank, world, port, semiring, transpose, iterations, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, tgt = graph()
        rng = np.random.default_rng(3)
        x = torch.from_numpy(rng.random(N))
        y = torch.zeros(N, dtype=torch.float64)
        parts = HostSpmvParts(off, tgt, semiring, transpose)
        res = spmv_iterate(parts, x, y, iterations)
        np.save(out + f"_{rank}.npy", res.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("semiring,transpose,iterations", [(0, False, 1), (1, True, 3)])
def test_gloo_ranks_equal_the_unpartitioned_products(tmp_path, semiring, transpose, iterations):
    out = str(tmp_path / "spmv")
    mp.start_processes(_spmv_rank, args=(2, _free_port(), semiring, transpose, iterations, out),
                       nprocs=2, start_method="spawn")
    off, tgt = graph()
    og = O.Graph.from_csr(N, off, tgt)
    x = np.random.default_rng(3).random(N)
    for _ in range(iterations):
        y = np.zeros(N)
        assert O.product(og, semiring, x, y, transpose=transpose) == 0
        x = y
    for rank in range(2):
        assert np.array_equal(np.load(out + f"_{rank}.npy"), x)
