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
