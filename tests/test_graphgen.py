"""The benchmark graphs: the oracle's copy of the generator (which the CPU
baseline uses, so that it never maps the CUDA library) gives the same CSR
as the CUDA library's, at a small scale and at the benchmark's scale 22."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W


@pytest.mark.parametrize("scale", [12, 22])
def test_oracle_and_library_generate_the_same_rmat(scale):
    a, b = O.rmat(scale), W.rmat(scale)
    assert a.id_space == b.id_space == 1 << scale
    assert np.array_equal(a.offsets, b.offsets)
    assert np.array_equal(a.targets, b.targets)
    if scale == 22:
        assert a.edges == 65_241_322  # the edge count the benchmark records


def test_oracle_and_library_generate_the_same_gnm():
    a, b = O.gnm(5000, 40000, seed=3), W.gnm(5000, 40000, seed=3)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.targets, b.targets)


def test_the_references_batched_shape_equals_its_per_source_search():
    # The CPU baseline's second arm: multi_source.rs's 64-sources-a-word push
    # (restated in the oracle, with per-source caps) gives the per-source
    # LevelSearch's depths and edges_traversed, repeated sources and caps of
    # 0 included, over a width that is not a multiple of 64.
    g = O.rmat(14, seed=3)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, reverse=False)
    rng = np.random.default_rng(4)
    src = rng.integers(0, g.id_space, 150).astype(np.uint64)
    src[10] = src[70] = src[3]
    caps = rng.integers(0, 17, 150).astype(np.uint32)
    caps[4] = 0
    a, ea = O.bfs_depths(og, src, caps)
    b, eb = O.bfs_depths_batched64(og, src, caps)
    assert np.array_equal(a, b) and np.array_equal(ea, eb)
