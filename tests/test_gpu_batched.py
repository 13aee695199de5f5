"""The batched searches against the oracle's per-source searches: depths
bit-exact, and per source the edges a push-only bfs traverses."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu


def graph(scale, seed=1):
    g = W.rmat(scale, seed=seed)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, reverse=False)
    return g, og, W.GraphVersion(g.offsets, g.targets)


@pytest.mark.parametrize("width", [1, 64, 100, 1024, 1500])
def test_bfs_batched_equals_per_source_bfs(width):
    g, og, gv = graph(14 if width > 200 else 16)
    rng = np.random.default_rng(width)
    src = rng.integers(0, g.id_space, width).astype(np.uint64)
    src[: min(3, width)] = src[0]  # repeated sources are searched apart
    caps = rng.integers(0, 17, width).astype(np.uint32)
    d, e = W.bfs_batched(gv, src, caps)
    do, eo = O.bfs_depths(og, src, caps)
    assert np.array_equal(d, do)
    assert np.array_equal(e, eo)


def test_bfs_batched_autotuned_schedules_agree():
    g, og, gv = graph(15)
    rng = np.random.default_rng(3)
    src = rng.integers(0, g.id_space, 300).astype(np.uint64)
    caps = rng.integers(1, 17, 300).astype(np.uint32)
    do, eo = O.bfs_depths(og, src, caps)
    s = W.autotune(gv, "bfs", 300)
    assert s.columns_per_pass in (32, 64, 128, 256, 512)
    d, e = W.bfs_batched(gv, src, caps)
    assert np.array_equal(d, do) and np.array_equal(e, eo)


def test_bfs_batched_device_outputs():
    torch = pytest.importorskip("torch")
    g, og, gv = graph(13)
    src = np.arange(0, 64, dtype=np.uint64) * 7
    caps = np.full(64, 16, np.uint32)
    d = torch.empty((64, g.id_space), dtype=torch.uint8, device="cuda")
    e = torch.empty(64, dtype=torch.int64, device="cuda")
    W.bfs_batched(gv, src, caps, depth_out=d, edges_out=e)
    do, eo = O.bfs_depths(og, src, caps)
    assert np.array_equal(d.cpu().numpy(), do)
    assert np.array_equal(e.cpu().numpy().astype(np.uint64), eo)
