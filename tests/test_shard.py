"""The sharded batched search's host side on two gloo ranks (CPU): each rank
runs its share of the sources (here through the oracle's per-source BFS)
into its rows of the output, the rows are broadcast from their owners, and
every rank's output equals the unsharded run."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import torch

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


def _search_into(og, sources, caps, depths, edges):
    def search(b, e):
        d, x = O.bfs_depths(og, sources[b:e], caps[b:e])
        depths[b:e] = torch.from_numpy(d)
        edges[b:e] = torch.from_numpy(x.astype(np.int64))
    return search


def _rank(rank, world, port, sources, caps, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        og = _graph()
        depths = torch.full((len(sources), og.n), 7, dtype=torch.uint8)
        edges = torch.full((len(sources),), -1, dtype=torch.int64)
        b, e = run_sharded(len(sources), _search_into(og, sources, caps, depths, edges),
                           [depths, edges])
        np.save(out + f"_{rank}_d.npy", depths.numpy())
        np.save(out + f"_{rank}_e.npy", edges.numpy())
        np.save(out + f"_{rank}_share.npy", np.array([b, e]))
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
    for rank in range(2):
        assert np.array_equal(np.load(out + f"_{rank}_d.npy"), do)
        assert np.array_equal(np.load(out + f"_{rank}_e.npy"), eo.astype(np.int64))
    assert [tuple(np.load(out + f"_{r}_share.npy")) for r in range(2)] == [(0, 19), (19, 37)]


def test_without_a_process_group_the_call_is_unsharded():
    og = _graph()
    sources = np.array([1, 2, 3], np.uint64)
    caps = np.array([2, 3, 4], np.uint32)
    d = torch.zeros((3, og.n), dtype=torch.uint8)
    e = torch.zeros(3, dtype=torch.int64)
    assert run_sharded(3, _search_into(og, sources, caps, d, e), [d, e]) == (0, 3)
    do, eo = O.bfs_depths(og, sources, caps)
    assert np.array_equal(d.numpy(), do) and np.array_equal(e.numpy(), eo.astype(np.int64))


def _wgraph():
    rng = np.random.default_rng(12)
    n = 200
    edges = [(0, int(a), int(b), float(rng.integers(1, 9)))
             for a, b in rng.integers(0, n, (1500, 2)) if a != b]
    return O.Graph.from_edges(n, edges, weighted=True, reverse=True)


def _rank_minplus(rank, world, port, sources, hops, out):
    # The min-plus shape of the sharded call (i64 distances and i32
    # iteration counts, two outputs of other widths), with the oracle's
    # sssp_vector loop as each rank's search; some ranks may own no rows.
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        og = _wgraph()
        dist_out = torch.full((len(sources), og.n), -7, dtype=torch.int64)
        its = torch.full((len(sources),), -1, dtype=torch.int32)

        def search(b, e):
            d, it = O.sssp_i64(og, sources[b:e], hops[b:e])
            dist_out[b:e] = torch.from_numpy(d)
            its[b:e] = torch.from_numpy(it.astype(np.int32))

        run_sharded(len(sources), search, [dist_out, its])
        np.save(out + f"_{rank}_d.npy", dist_out.numpy())
        np.save(out + f"_{rank}_i.npy", its.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("count", [2, 5])
def test_three_gloo_ranks_gather_minplus_rows_even_when_a_rank_owns_none(tmp_path, count):
    rng = np.random.default_rng(count)
    sources = rng.integers(0, 200, count).astype(np.uint64)
    hops = rng.integers(0, 12, count).astype(np.uint32)
    out = str(tmp_path / "m")
    mp.start_processes(_rank_minplus, args=(3, _free_port(), sources, hops, out), nprocs=3,
                       start_method="spawn")
    do, ito = O.sssp_i64(_wgraph(), sources, hops)
    for rank in range(3):
        assert np.array_equal(np.load(out + f"_{rank}_d.npy"), do)
        assert np.array_equal(np.load(out + f"_{rank}_i.npy"), ito.astype(np.int32))
