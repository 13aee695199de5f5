"""Closeness and harmonic centrality on the batched BFS against the oracle's
restatement of the reference's batched measures: bit-exact (the integer
totals are exact and the harmonic sums are added in the reference's order:
batch of 64 sources, then distance)."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu


def both(og, gv, sampling, tomb=None, columns=0):
    src = W.sample_sources(gv.id_space, sampling, tomb)
    out = []
    for measure in ("closeness", "harmonic"):
        for wf in ((True, False) if measure == "closeness" else (False,)):
            if measure == "closeness":
                got = W.closeness_centrality(gv, sampling, wf, tomb, columns)
            else:
                got = W.harmonic_centrality(gv, sampling, tomb, columns)
            assert got.sources == len(src)
            want = O.centrality(og, measure, src, tombstones=tomb, wf_improved=wf)
            out.append((measure, wf, got.values, want))
    return out


def test_the_reference_example():
    # compute/centrality/tests.rs:117-143.
    pairs = [(0, 1), (1, 2), (2, 3), (0, 2), (3, 0), (1, 3), (4, 1)]
    og = O.Graph.from_edges(5, [(0, s, t, 1.0) for s, t in pairs], weighted=False)
    off, tgt, _, _, _, _ = og.csr()
    gv = W.GraphVersion(off, tgt)
    c = W.closeness_centrality(gv)
    assert np.allclose(c.values, [0.5, 4 / 7, 2 / 3, 2 / 3, 0.0], rtol=1e-15, atol=0)
    h = W.harmonic_centrality(gv)
    assert np.allclose(h.values, [7 / 3, 17 / 6, 3, 3, 0], rtol=1e-15, atol=0)
    h2 = W.harmonic_centrality(gv, W.Sampling(population=np.array([1, 0, 1, 0, 0])))
    assert h2.sources == 2
    assert np.allclose(h2.values, [2.0, 8 / 3, 4.0, 3.0, 0.0], rtol=1e-15, atol=0)


@pytest.mark.parametrize("columns,k", [(64, None), (128, 300), (1024, None), (256, 1000)])
def test_rmat_every_node_and_samples(columns, k):
    g = W.rmat(11, seed=5)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    rng = np.random.default_rng(columns)
    tomb = W.node_set(g.id_space, rng.integers(0, g.id_space, 20)) if k else None
    for measure, wf, got, want in both(og, gv, W.Sampling(k=k, seed=11), tomb, columns):
        assert got.tobytes() == want.tobytes(), (measure, wf)


def test_deep_graphs_run_their_passes_deeper():
    # A path of 300 nodes beside a random graph: searches of ~300 levels,
    # past the first 32 and 64 levels a pass tries.
    rng = np.random.default_rng(2)
    n = 700
    pairs = [(i, i + 1) for i in range(299)]
    pairs += [(int(a), int(b)) for a, b in rng.integers(300, n, (2000, 2)) if a != b]
    pairs += [(299, 300), (650, 0)]
    og = O.Graph.from_edges(n, [(0, s, t, 1.0) for s, t in pairs], weighted=False)
    off, tgt, _, _, _, _ = og.csr()
    gv = W.GraphVersion(off, tgt)
    for measure, wf, got, want in both(og, gv, W.Sampling(k=150, seed=4), None, 64):
        assert got.tobytes() == want.tobytes(), (measure, wf)


def test_searches_deeper_than_the_limit_are_refused():
    n = 1100
    off = np.arange(n + 1, dtype=np.uint64)
    off[-1] = n - 1
    tgt = np.arange(1, n, dtype=np.uint32)
    gv = W.GraphVersion(off, tgt)
    with pytest.raises(W.api.Unsupported):
        W.closeness_centrality(gv, W.Sampling(population=np.eye(1, n, 0, dtype=np.uint8)[0]),
                               columns_per_pass=64)


def test_no_sources_gives_zeros():
    g = W.rmat(8, seed=1)
    gv = W.GraphVersion(g.offsets, g.targets)
    empty = W.Sampling(population=np.zeros(g.id_space, np.uint8))
    assert not W.closeness_centrality(gv, empty).values.any()
    assert not W.harmonic_centrality(gv, empty).values.any()
