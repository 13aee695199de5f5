"""The PageRank adjoint against the FP64 CPU adjoint and central finite
differences (step 1e-6) of the forward solve; top_k against the oracle."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu


def weighted_rmat(scale, seed=1):
    g = W.rmat(scale, seed=seed)
    w = W.edge_weights(g, "lognormal")
    return g, w


def test_adjoint_matches_the_cpu_adjoint():
    g, w = weighted_rmat(11)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w)
    gv = W.GraphVersion(g.offsets, g.targets, w)
    rng = np.random.default_rng(2)
    losses = [rng.choice(g.id_space, 100, replace=False) for _ in range(40)]
    pr = W.PageRank(0.85, None, 150)
    grad, ranks, it = W.pagerank_adjoint(gv, losses, pr, adjoint_tol=1e-15)
    go, ro, ito = O.pagerank_adjoint(og, losses, 0.85, None, 150, 1e-15)
    assert np.abs(ranks - ro).sum() / ro.sum() <= 1e-12
    scale = np.abs(go).max()
    assert np.abs(grad - go).max() <= 1e-9 * scale


def test_adjoint_matches_central_finite_differences():
    g, w = weighted_rmat(9, seed=3)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w)
    gv = W.GraphVersion(g.offsets, g.targets, w)
    rng = np.random.default_rng(4)
    targets = rng.choice(g.id_space, 60, replace=False)
    grad, _, _ = W.pagerank_adjoint(gv, [targets], W.PageRank(0.85, None, 300),
                                    adjoint_tol=1e-16)
    h = 1e-6
    checked = 0
    for e in rng.choice(g.edges, 40, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[e] += h
        wm[e] -= h
        lp = O.pagerank(O.Graph.from_csr(g.id_space, g.offsets, g.targets, wp), 0.85, None, 300)[0]
        lm = O.pagerank(O.Graph.from_csr(g.id_space, g.offsets, g.targets, wm), 0.85, None, 300)[0]
        fd = (lp[targets].sum() - lm[targets].sum()) / (2 * h)
        # Relative to the gradient, or to the FD's own rounding floor.
        floor = 1e-16 * lp[targets].sum() / h
        assert abs(fd - grad[0, e]) <= 1e-6 * abs(grad[0, e]) + 4 * floor, (e, fd, grad[0, e])
        checked += 1
    assert checked == 40


def test_top_k_matches_the_oracle():
    g = W.rmat(12)
    gv = W.GraphVersion(g.offsets, g.targets)
    rng = np.random.default_rng(5)
    x = rng.integers(0, 50, g.id_space).astype(np.float64)
    x[rng.integers(0, g.id_space, 20)] = np.nan
    x[3] = -0.0
    x[4] = 0.0
    tomb = O.tombstone_words(g.id_space, rng.integers(0, g.id_space, 300))
    for desc in (True, False):
        for k in (1, 10, 1000, g.id_space + 5):
            got = W.top_k(gv, x, k, desc, tomb)
            nodes, vals = O.topk(x, k, desc, tomb)
            assert [a for a, _ in got] == list(nodes)
