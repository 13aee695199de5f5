"""Betweenness centrality on the batched BFS (wc_betweenness) against the
oracle's restatement of the reference's one-source-at-a-time Brandes: the
reference's known answers, and R-MAT graphs bit for bit while no row has
over 256 entries (path counts stay far below 2^53 here), within 1e-13
relative where a long row's pieces are summed in order.""" 

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu

from test_oracle_kats import BETWEENNESS_KATS


def test_the_reference_example():
    pairs = [(0, 1), (1, 2), (2, 3), (0, 2), (3, 0), (1, 3)]
    og = O.Graph.from_edges(5, [(0, s, t, 1.0) for s, t in pairs], weighted=False)
    off, tgt, _, _, _, _ = og.csr()
    gv = W.GraphVersion(off, tgt)
    two = W.Sampling(population=np.array([1, 0, 1, 0, 0]))
    for normalized, endpoints, exact, from_two in BETWEENNESS_KATS:
        got = W.betweenness_centrality(gv, normalized=normalized, endpoints=endpoints)
        assert np.allclose(got.values, exact, rtol=1e-12, atol=0)
        got = W.betweenness_centrality(gv, two, normalized=normalized, endpoints=endpoints)
        assert got.sources == 2
        assert np.allclose(got.values, from_two, rtol=1e-12, atol=0)


@pytest.mark.parametrize("scale,k,endpoints", [(9, None, False), (10, 100, True),
                                               (11, 150, False)])
def test_rmat_matches_the_oracle_bit_for_bit(scale, k, endpoints):
    g = W.rmat(scale, seed=scale)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    rng = np.random.default_rng(scale)
    tomb = W.node_set(g.id_space, rng.integers(0, g.id_space, 5)) if k else None
    src = W.sample_sources(g.id_space, W.Sampling(k=k, seed=3), tomb)
    for normalized in (True, False):
        got = W.betweenness_centrality(gv, normalized=normalized, endpoints=endpoints,
                                       tombstones=tomb, sources=src)
        want = O.betweenness(og, src, tombstones=tomb, normalized=normalized, endpoints=endpoints)
        if np.diff(g.offsets.astype(np.int64)).max() <= 256:
            assert got.values.tobytes() == want.tobytes(), normalized
        else:  # rows over 256 entries sum their pieces in order: reassociated
            assert np.allclose(got.values, want, rtol=1e-13, atol=0), normalized


def test_undirected_deep_graph():
    # A symmetrised path of 200 nodes beside a random part: searches past
    # the first 32 and 64 levels; directed=False halves the rescale.
    rng = np.random.default_rng(4)
    n = 400
    pairs = [(i, i + 1) for i in range(199)]
    pairs += [(int(a), int(b)) for a, b in rng.integers(200, n, (800, 2)) if a != b]
    pairs += [(199, 200)]
    pairs += [(b, a) for a, b in pairs]
    og = O.Graph.from_edges(n, [(0, s, t, 1.0) for s, t in pairs], weighted=False)
    off, tgt, _, _, _, _ = og.csr()
    gv = W.GraphVersion(off, tgt)
    src = W.sample_sources(n, W.Sampling(k=70, seed=1))
    got = W.betweenness_centrality(gv, directed=False, sources=src)
    want = O.betweenness(og, src, directed=False)
    assert got.values.tobytes() == want.tobytes()
