"""Row-partitioned PageRank over several GPUs (one process per GPU).

The single-source solve of compute/pagerank/mod.rs:96-151 with its rows cut
into one range per rank (the library's `wc_pagerank_part_*` entry points
cut the locality-ordered reverse CSR into ranges of about equal entries).
Every rank holds the whole version and, each iteration, pulls its own rows;
then the ranks exchange what the next iteration reads:

- an all-reduce (sum) of two scalars, the parts' L1 changes and their next
  dangling ranks, from which every rank takes the same stop decision;
- an all-gather of the parts' rows of the next message vector (each part's
  rows broadcast from it into the same rows on every rank), 8·n bytes.

After the last iteration the parts' rows of the rank vector are gathered
the same way and renumbered into dense-id order.  The collectives go over
the caller's process group (`nccl` between GPUs; `gloo` on the host, where
the tests drive the same loop with a host implementation of the parts).
"""

from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _abi as A


class DeviceParts:
    """A rank's part of the solve on its GPU, through the C ABI.  ranks2 /
    messages2: the rank and message vectors of even and odd iterations
    (torch float64, 2 × id_space, on this rank's device), which the driver
    exchanges rows of."""

    def __init__(self, graph, tombstones=None, pagerank=None, stream=None):
        import torch

        from .api import PageRank, _call, _pr_opts, _ptr, _raise

        self.graph = graph
        self.pagerank = pagerank or PageRank()
        self._call, self._raise, self._ptr = _call, _raise, _ptr
        self.tombstones = tombstones
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        n = graph.id_space
        self.ranks2 = torch.empty((2, n), dtype=torch.float64, device="cuda")
        self.messages2 = torch.empty((2, n), dtype=torch.float64, device="cuda")
        self.opts, _ = _pr_opts(self.pagerank)

    def rows(self, parts: int) -> np.ndarray:
        b = np.zeros(parts + 1, np.uint64)
        self._raise(A.load().wc_pagerank_part_rows(self.graph.handle, parts, self._ptr(b)),
                    A.ErrorDetail())
        return b.astype(np.int64)

    def begin(self, parts: int, part: int) -> A.PageRankPartInfo:
        info = A.PageRankPartInfo()
        call, detail = self._call(None, self.stream)
        self._raise(A.load().wc_pagerank_part_begin(
            self.graph.handle, C.byref(call), C.byref(self.opts), self._ptr(self.tombstones),
            parts, part, self.ranks2.data_ptr(), self.messages2.data_ptr(), C.byref(info)),
            detail)
        return info

    def step(self, iteration: int, dangling: float):
        sums = (C.c_double * 2)()
        call, detail = self._call(None, self.stream)
        self._raise(A.load().wc_pagerank_part_step(self.graph.handle, C.byref(call), iteration,
                                                   dangling, sums), detail)
        return sums[0], sums[1]

    def end(self, iterations: int, out=None):
        ranks = out if out is not None else np.zeros(self.graph.id_space, np.float64)
        call, detail = self._call(None, self.stream)
        self._raise(A.load().wc_pagerank_part_end(self.graph.handle, C.byref(call), iterations,
                                                  self._ptr(ranks)), detail)
        return ranks


def _broadcast_rows(t, bounds: Sequence[int], group=None) -> None:
    """Each part r's rows [bounds[r], bounds[r + 1]) of the 1-D tensor `t`
    broadcast from rank r into the same rows on every rank."""
    import torch.distributed as dist

    for r in range(len(bounds) - 1):
        b, e = int(bounds[r]), int(bounds[r + 1])
        if e > b:
            src = dist.get_global_rank(group, r) if group is not None else r
            dist.broadcast(t[b:e], src=src, group=group)


def solve(parts, max_iter: int, has_tol: bool, group=None, out=None, collective_device=None):
    """The partitioned solve's loop on this rank over `parts` (DeviceParts,
    or a host implementation of the same methods: rows, begin, step, end,
    and the ranks2 / messages2 tensors).  Without an initialised process
    group it is one part.  Returns (ranks in dense-id order, iterations)."""
    import torch
    import torch.distributed as dist

    grouped = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if grouped else 1
    rank = dist.get_rank(group) if grouped else 0
    bounds = parts.rows(world)
    info = parts.begin(world, rank)
    dev = collective_device if collective_device is not None else parts.messages2.device
    dangling, iterations = info.dangling, 0
    for it in range(max_iter):
        delta, nxt = parts.step(it, dangling)
        if grouped:
            sums = torch.tensor([delta, nxt], dtype=torch.float64, device=dev)
            dist.all_reduce(sums, group=group)
            delta, nxt = sums.tolist()
            _broadcast_rows(parts.messages2[(it + 1) & 1], bounds, group)
        iterations = it + 1
        dangling = nxt
        # The stop test of pagerank/mod.rs:141-147 on the summed change.
        if has_tol and delta < info.threshold:
            break
    if grouped:
        _broadcast_rows(parts.ranks2[iterations & 1], bounds, group)
    return parts.end(iterations, out), iterations


def pagerank_partitioned(graph, tombstones=None, pagerank=None, group=None, out=None):
    """`pagerank` with its rows partitioned over the ranks of `group`, one
    GPU each (every rank calls it with its own upload of the version).
    Returns Ranks as `pagerank` does, on every rank."""
    from .api import PageRank, Ranks

    pr = pagerank or PageRank()
    parts = DeviceParts(graph, tombstones, pr)
    ranks, iterations = solve(parts, pr.max_iter, pr.tol is not None, group, out)
    return Ranks(ranks, iterations)


# ------------------------------------------------------------------ products


class SpmvDeviceParts:
    """A rank's part of a row-partitioned product on its GPU, through the C
    ABI: wc_spmv_part computes the part's rows of y = A ⊗ x (or Aᵀ ⊗ x)
    from the whole x, leaving y's other rows as they are."""

    def __init__(self, graph, product, stream=None):
        from .api import _call, _dtype, _product_c, _ptr, _raise

        self.graph, self.product = graph, product
        self._call, self._dtype, self._ptr, self._raise = _call, _dtype, _ptr, _raise
        self.pc, self._mask = _product_c(product)
        # torch's stream: the collectives between products are ordered on it.
        if stream is None:
            import torch
            stream = torch.cuda.current_stream()
        self.stream = stream

    def rows(self, parts: int) -> np.ndarray:
        b = np.zeros(parts + 1, np.uint64)
        self._raise(A.load().wc_spmv_part_rows(self.graph.handle, int(self.product.transpose),
                                               parts, self._ptr(b)), A.ErrorDetail())
        return b.astype(np.int64)

    def apply(self, parts: int, part: int, x, y) -> None:
        call, detail = self._call(None, self.stream)
        self._raise(A.load().wc_spmv_part(self.graph.handle, C.byref(call), C.byref(self.pc),
                                          self._dtype(y), parts, part, self._ptr(x),
                                          self._ptr(y)), detail)


def spmv_iterate(parts, x, y, iterations: int = 1, group=None):
    """`iterations` products y = A ⊗ x with the rows partitioned over the
    ranks of `group`, each product's y gathered on every rank (its parts'
    rows broadcast from their owners) and becoming the next x.  `parts`:
    SpmvDeviceParts, or a host implementation of rows / apply.  x and y are
    1-D tensors of id_space elements (device tensors over NCCL, host ones
    over gloo); returns the last product's vector (x or y)."""
    import torch.distributed as dist

    grouped = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if grouped else 1
    rank = dist.get_rank(group) if grouped else 0
    bounds = parts.rows(world)
    for _ in range(iterations):
        parts.apply(world, rank, x, y)
        if grouped:
            _broadcast_rows(y, bounds, group)
        x, y = y, x
    return x


def spmv_partitioned(graph, product, x, y, group=None, iterations: int = 1):
    """`spmv` with its rows partitioned over the ranks of `group`, one GPU
    each (every rank calls it with its own upload of the version and the
    same x).  y (and, past one iteration, x) is overwritten; returns the
    tensor holding the result, the same on every rank."""
    return spmv_iterate(SpmvDeviceParts(graph, product), x, y, iterations, group)


# ------------------------------------------------------------------ searches


class BfsDeviceParts:
    """A rank's part of a row-partitioned level search on its GPU, through
    the C ABI.  frontier2: the frontiers of even and odd levels (torch int64,
    2 × words, on this rank's device), whose words the driver exchanges;
    depth: the depths (torch int32 view of u32, WC_UNREACHED as -1) into
    which the part's rows are written at the end."""

    def __init__(self, graph, starts, max_depth=None, direction: str = "out", stream=None):
        import torch

        from .api import _DIRECTIONS, _call, _ptr, _raise

        self.graph = graph
        self._call, self._ptr, self._raise = _call, _ptr, _raise
        self.direction = _DIRECTIONS[direction]
        self.starts = np.ascontiguousarray(np.asarray(starts, dtype=np.uint64))
        self.max_depth = A.UNREACHED if max_depth is None else int(max_depth)
        # torch's stream: the collectives between levels are ordered on it.
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        n = graph.id_space
        self.words = (n + 63) // 64
        self.frontier2 = torch.zeros(2 * max(self.words, 1), dtype=torch.int64, device="cuda")
        self.depth = torch.full((n,), -1, dtype=torch.int32, device="cuda")

    def frontier(self, level: int):
        h = (level & 1) * self.words
        return self.frontier2[h: h + self.words]

    def rows(self, parts: int) -> np.ndarray:
        b = np.zeros(parts + 1, np.uint64)
        self._raise(A.load().wc_bfs_part_rows(self.graph.handle, self.direction, parts,
                                              self._ptr(b)), A.ErrorDetail())
        return b.astype(np.int64)

    def begin(self, parts: int, part: int) -> A.BfsPartInfo:
        info = A.BfsPartInfo()
        call, detail = self._call(None, self.stream)
        self._raise(A.load().wc_bfs_part_begin(
            self.graph.handle, C.byref(call), self.direction, self._ptr(self.starts),
            len(self.starts), self.max_depth, parts, part, self.frontier2.data_ptr(),
            C.byref(info)), detail)
        return info

    def step(self, level: int, frontier_edges: int):
        sums = (C.c_uint64 * 2)()
        call, detail = self._call(None, self.stream)
        self._raise(A.load().wc_bfs_part_step(self.graph.handle, C.byref(call), level,
                                              frontier_edges, sums), detail)
        return int(sums[0]), int(sums[1])

    def end(self):
        call, detail = self._call(None, self.stream)
        self._raise(A.load().wc_bfs_part_end(self.graph.handle, C.byref(call),
                                             self.depth.data_ptr()), detail)
        return self.depth


def search(parts, max_depth=None, group=None):
    """The partitioned level search's loop on this rank over `parts`
    (BfsDeviceParts, or a host implementation of rows, begin, step, end,
    frontier and the frontier2 / depth tensors).  Each level: the parts
    reach their rows, the ranks sum the next frontier's nodes and out-edges
    (one all-reduce of two integers, from which every rank takes the same
    decisions) and gather its words (each part's words broadcast from it).
    The search stops when the frontier is empty or at max_depth.  Returns
    (depth tensor gathered on every rank, levels run)."""
    import torch
    import torch.distributed as dist

    grouped = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if grouped else 1
    rank = dist.get_rank(group) if grouped else 0
    bounds = parts.rows(world)
    word_bounds = [(int(b) + 63) // 64 for b in bounds]
    info = parts.begin(world, rank)
    count, edges = int(info.frontier), int(info.frontier_edges)
    level = 0
    while count and (max_depth is None or level < max_depth):
        count, edges = parts.step(level, edges)
        if grouped:
            sums = torch.tensor([count, edges], dtype=torch.int64, device=parts.frontier2.device)
            dist.all_reduce(sums, group=group)
            count, edges = (int(v) for v in sums.tolist())
            _broadcast_rows(parts.frontier(level + 1), word_bounds, group)
        level += 1
    depth = parts.end()
    if grouped:
        _broadcast_rows(depth, bounds, group)
    return depth, level


def bfs_partitioned(graph, starts, max_depth=None, direction: str = "out", group=None):
    """The depths of `bfs_depths` with the rows partitioned over the ranks
    of `group`, one GPU each (every rank calls it with its own upload of the
    version and the same starts).  Returns (depth u32[id_space] on the host,
    WC_UNREACHED where not reached; levels run), the same on every rank."""
    parts = BfsDeviceParts(graph, starts, max_depth, direction)
    depth, levels = search(parts, max_depth, group)
    return depth.cpu().numpy().view(np.uint32), levels
