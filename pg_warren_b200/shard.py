"""Sharding the batched searches over ranks (one process per GPU).

The batched searches (`bfs_batched`, `minplus_batched`, `ppr_batched`)
shard by column: every rank holds the whole version and runs a contiguous
share of the sources (or seed sets); nothing is exchanged while they run.
The only collective is the gather of the per-source results at the end,
over the process group the caller set up (`nccl` between GPUs, `gloo` on
the host).  Single-source calls (SpMV, PageRank, BFS, Lanczos) run as
replicas.
"""

from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np


def shard_range(count: int, world: int, rank: int) -> Tuple[int, int]:
    """The [begin, end) of `count` columns that `rank` of `world` runs:
    contiguous, sizes differing by at most one, lower ranks first."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(count, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def run_sharded(sources: Sequence[int], max_depths: Sequence[int],
                search: Callable[[np.ndarray, np.ndarray], Tuple[np.ndarray, np.ndarray]],
                group=None, gather_depths: bool = True):
    """Runs `search(sources_share, caps_share) -> (depths u8[k, n], edges
    u64[k])` on this rank's share of the columns and gathers the results to
    every rank, in source order: (depths or None, edges).  Without an
    initialised process group it is the unsharded call."""
    import torch.distributed as dist

    src = np.ascontiguousarray(np.asarray(sources, dtype=np.uint64))
    caps = np.ascontiguousarray(np.asarray(max_depths, dtype=np.uint32))
    if not (dist.is_available() and dist.is_initialized()):
        d, e = search(src, caps)
        return (d if gather_depths else None), np.asarray(e, dtype=np.uint64)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b, e_ = shard_range(len(src), world, rank)
    d, e = search(src[b:e_], caps[b:e_])
    part = {"edges": np.asarray(e, dtype=np.uint64),
            "depths": np.asarray(d) if gather_depths else None}
    parts: list = [None] * world
    dist.all_gather_object(parts, part, group=group)
    edges = np.concatenate([p["edges"] for p in parts]) if parts else np.zeros(0, np.uint64)
    depths: Optional[np.ndarray] = None
    if gather_depths:
        depths = np.concatenate([p["depths"] for p in parts], axis=0)
    return depths, edges


def bfs_batched_sharded(graph, sources, max_depths, group=None, gather_depths: bool = True):
    """`bfs_batched` with the sources sharded over the ranks of `group`."""
    from .api import bfs_batched

    return run_sharded(sources, max_depths, lambda s, c: bfs_batched(graph, s, c), group,
                       gather_depths)
