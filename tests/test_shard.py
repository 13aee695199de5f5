"""The sharded batched search's host side on two gloo ranks (CPU): each rank
runs its share of the sources (here through the oracle's per-source BFS)
and the gathered depths and edge counts equal the unsharded run."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from pg_warren_b200.shard import run_sharded, shard_range


def test_shard_range_covers_every_column_once():
    for count in (0, 1, 7, 1024, 1025):
        for world in (1, 2, 3, 8):
            spans = [shard_range(count, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _graph():
    rng = np.random.default_rng(11)
    n = 300
    edges = [(0, int(a), int(b), 1.0) for a, b in rng.integers(0, n, (2000, 2)) if a != b]
    return O.Graph.from_edges(n, edges, weighted=False, reverse=False)


def _rank(rank, world, port, sources, caps, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        og = _graph()
        depths, edges = run_sharded(sources, caps, lambda s, c: O.bfs_depths(og, s, c))
        if rank == 0:
            np.save(out + "_d.npy", depths)
            np.save(out + "_e.npy", edges)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_the_unsharded_result(tmp_path):
    rng = np.random.default_rng(5)
    sources = rng.integers(0, 300, 37).astype(np.uint64)
    caps = rng.integers(0, 9, 37).astype(np.uint32)
    out = str(tmp_path / "r")
    mp.start_processes(_rank, args=(2, _free_port(), sources, caps, out), nprocs=2,
                       start_method="spawn")
    do, eo = O.bfs_depths(_graph(), sources, caps)
    assert np.array_equal(np.load(out + "_d.npy"), do)
    assert np.array_equal(np.load(out + "_e.npy"), eo)


def test_without_a_process_group_the_call_is_unsharded():
    og = _graph()
    sources = np.array([1, 2, 3], np.uint64)
    caps = np.array([2, 3, 4], np.uint32)
    d, e = run_sharded(sources, caps, lambda s, c: O.bfs_depths(og, s, c))
    do, eo = O.bfs_depths(og, sources, caps)
    assert np.array_equal(d, do) and np.array_equal(e, eo)
