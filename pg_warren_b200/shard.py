"""Sharding the batched searches over ranks (one process per GPU).

The batched searches (`bfs_batched`, `minplus_batched`, `ppr_batched`)
shard by column: every rank holds the whole version and runs a contiguous
share of the sources (or seed sets) into its rows of the caller's output;
nothing is exchanged while they run.  The one collective is the gather at
the end: each rank's rows are broadcast from it into the same rows of every
other rank's output (`nccl` between GPUs, over NVLink; `gloo` for host
tensors), so the results land in the caller's buffers with no staging copy
and no serialisation.  Single-source calls run over the row partition of
`partition.py`, or as replicas.
"""

from __future__ import annotations

from typing import Callable, Sequence, Tuple

import numpy as np


def shard_range(count: int, world: int, rank: int) -> Tuple[int, int]:
    """The [begin, end) of `count` columns that `rank` of `world` runs:
    contiguous, sizes differing by at most one, lower ranks first."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(count, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def _group():
    import torch.distributed as dist

    return dist.is_available() and dist.is_initialized()


def gather_rows(outputs: Sequence, count: int, group=None) -> None:
    """Every rank's rows [begin, end) (shard_range of `count`) of each tensor
    in `outputs` (first dimension: the columns) broadcast from that rank into
    the same rows on every rank.  The same calls in the same order on every
    rank; a rank with no rows skips none of them."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    for r in range(world):
        b, e = shard_range(count, world, r)
        if e == b:
            continue
        for t in outputs:
            view = t[b:e]
            assert view.is_contiguous(), "each rank's rows must be contiguous"
            dist.broadcast(view, src=dist.get_global_rank(group, r) if group is not None else r,
                           group=group)


def run_sharded(count: int, search: Callable[[int, int], None], outputs: Sequence,
                group=None, gather: bool = True) -> Tuple[int, int]:
    """Runs `search(begin, end)` for this rank's share of `count` columns
    (it fills rows [begin, end) of `outputs`), then gathers every rank's rows
    into every rank's `outputs` (unless `gather` is false).  Without an
    initialised process group it is the unsharded call.  Returns this rank's
    (begin, end)."""
    import torch.distributed as dist

    if not _group():
        search(0, count)
        return 0, count
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b, e = shard_range(count, world, rank)
    if e > b:
        search(b, e)
    if gather:
        gather_rows(outputs, count, group)
    return b, e


def bfs_batched_sharded(graph, sources, max_depths, depth_out, edges_out, group=None,
                        gather: bool = True, stream=None):
    """`bfs_batched` with the sources sharded over the ranks of `group`:
    depth_out (u8[k, n]) and edges_out (i64[k]) are this rank's device (or,
    with gloo, host) tensors, filled for every source once gathered."""
    from .api import bfs_batched

    src = np.ascontiguousarray(np.asarray(sources, dtype=np.uint64))
    caps = np.ascontiguousarray(np.asarray(max_depths, dtype=np.uint32))

    def search(b, e):
        bfs_batched(graph, src[b:e], caps[b:e], depth_out=depth_out[b:e],
                    edges_out=edges_out[b:e], stream=stream)

    return run_sharded(len(src), search, [depth_out, edges_out], group, gather)


def minplus_batched_sharded(graph, sources, max_hops, dist_out, iterations_out, group=None,
                            gather: bool = True):
    """`minplus_batched` with the sources sharded: dist_out i64[k, n] and
    iterations_out i32[k] filled for every source once gathered."""
    from .api import minplus_batched

    src = np.ascontiguousarray(np.asarray(sources, dtype=np.uint64))
    hops = np.ascontiguousarray(np.asarray(max_hops, dtype=np.uint32))

    def search(b, e):
        minplus_batched(graph, src[b:e], hops[b:e], dist_out=dist_out[b:e],
                        iterations_out=iterations_out[b:e])

    return run_sharded(len(src), search, [dist_out, iterations_out], group, gather)


def ppr_batched_sharded(graph, seed_sets, pagerank, ranks_out, iterations_out, group=None,
                        gather: bool = True):
    """`ppr_batched` with the seed sets sharded: ranks_out f64[k, n] and
    iterations_out i32[k] filled for every set once gathered."""
    from .api import ppr_batched

    sets = list(seed_sets)

    def search(b, e):
        ppr_batched(graph, sets[b:e], pagerank, ranks_out=ranks_out[b:e],
                    iterations_out=iterations_out[b:e])

    return run_sharded(len(sets), search, [ranks_out, iterations_out], group, gather)
