"""Parity of the CUDA path with the oracle: products, PageRank, traversal.

Bit-exact for integer, boolean, min/max and traversal results; floating-point
plus within the stated tolerance (rows over 256 entries and PageRank's sums
are reassociated): SpMV f64 plus to 1e-13 relative per row, PageRank to
1e-12 relative L1 with the same iteration count.
"""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu

SEMIRINGS = W.api.A.SEMIRINGS
I64_MAX = np.iinfo(np.int64).max


def random_graph(rng, n, m, weights="int", relations=1):
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    if weights == "int":
        w = rng.integers(-3, 5, m).astype(np.float64)
    elif weights == "pos":
        w = rng.integers(1, 100, m).astype(np.float64)
    else:
        w = rng.choice([0.1, 0.7, 1e-3, 3.0, -0.0, 2.5], m)
    edges = [(int(rng.integers(0, relations)), int(s), int(t), float(x))
             for s, t, x in zip(src, dst, w)]
    og = O.Graph.from_edges(n, edges, weighted=True, relations=relations)
    off, tgt, ww, _, _, _ = og.csr()
    return og, W.GraphVersion(off, tgt, ww), off, tgt, ww


def hub_graph(rng, n, hub_degree):
    # A few rows far over the 256-entry tile bound, split into 4096-entry
    # pieces, beside many short rows.
    pairs = set()
    for h in range(3):
        for t in rng.choice(n, hub_degree, replace=False):
            pairs.add((h, int(t)))
    for _ in range(5 * n):
        pairs.add((int(rng.integers(0, n)), int(rng.integers(0, n))))
    edges = [(0, s, t, float(rng.integers(1, 9))) for s, t in sorted(pairs)]
    og = O.Graph.from_edges(n, edges, weighted=True)
    off, tgt, ww, _, _, _ = og.csr()
    return og, W.GraphVersion(off, tgt, ww), off, tgt, ww


def values(rng, dtype, n, width=1):
    shape = (n,) if width == 1 else (n, width)
    if dtype == np.float64:
        return rng.integers(-4, 5, shape).astype(np.float64) * 0.5
    if dtype == np.int64:
        v = rng.integers(-4, 5, shape).astype(np.int64)
        v[rng.random(shape) < 0.1] = I64_MAX
        return v
    return (rng.random(shape) < 0.4).astype(np.uint8)


def run_both(og, gv, semiring, x, y0, **kw):
    yo = y0.copy()
    so = O.product(og, SEMIRINGS.index(semiring), x, yo, transpose=kw.get("transpose", False),
                   mask=kw.get("mask"), mask_dtype=1, complement=kw.get("complement", False),
                   replace=kw.get("replace", False),
                   accumulate=W.api.A.BINARY_OPS.index(kw["accumulate"]) if kw.get("accumulate") else -1)
    yg = y0.copy()
    p = W.Product(semiring, transpose=kw.get("transpose", False), mask=kw.get("mask"),
                  complement=kw.get("complement", False), replace=kw.get("replace", False),
                  accumulate=kw.get("accumulate"))
    try:
        (W.spmv if x.ndim == 1 else W.spmm)(gv, p, x, yg)
        sg = 0
    except W.api.WarrenError as e:
        sg = e.status
    return so, yo, sg, yg


@pytest.mark.parametrize("semiring", SEMIRINGS)
@pytest.mark.parametrize("dtype", [np.float64, np.int64, np.uint8])
def test_spmv_every_semiring_matches_the_oracle(semiring, dtype):
    rng = np.random.default_rng(SEMIRINGS.index(semiring) * 7 + 3)
    for graph in ("small", "hubs"):
        if graph == "small":
            og, gv, *_ = random_graph(rng, 300, 2000)
        else:
            og, gv, *_ = hub_graph(rng, 12000, 9000)
        n = gv.id_space
        for transpose in (False, True):
            x = values(rng, dtype, n)
            y0 = values(rng, dtype, n)
            so, yo, sg, yg = run_both(og, gv, semiring, x, y0, transpose=transpose)
            assert so == sg, (semiring, graph, transpose)
            if so:
                continue
            if dtype == np.float64 and semiring.startswith("plus"):
                assert np.allclose(yg, yo, rtol=1e-13, atol=1e-12)
                if graph == "small":  # rows under 256 entries fold in order
                    assert yg.tobytes() == yo.tobytes()
            else:
                assert yg.tobytes() == yo.tobytes(), (semiring, graph, transpose)


@pytest.mark.parametrize("accumulate", [None, "plus", "min", "max", "second"])
def test_spmv_mask_replace_accumulate(accumulate):
    rng = np.random.default_rng(11)
    og, gv, *_ = random_graph(rng, 500, 3000)
    for semiring in ("plus_times", "min_plus", "lor_land"):
        for complement in (False, True):
            for replace in (False, True):
                x = values(rng, np.float64, 500)
                y0 = values(rng, np.float64, 500)
                mask = (rng.random(500) < 0.5).astype(np.float64)
                mask[3] = np.nan
                so, yo, sg, yg = run_both(og, gv, semiring, x, y0, mask=mask, complement=complement,
                                          replace=replace, accumulate=accumulate, transpose=True)
                assert so == sg
                assert yg.tobytes() == yo.tobytes()


def test_spmm_matches_the_oracle():
    rng = np.random.default_rng(5)
    og, gv, *_ = random_graph(rng, 400, 2500, weights="pos")
    for semiring, dtype in (("min_plus", np.int64), ("plus_times", np.float64),
                            ("lor_land", np.uint8)):
        x = values(rng, dtype, 400, width=37)
        y0 = values(rng, dtype, 400, width=37)
        so, yo, sg, yg = run_both(og, gv, semiring, x, y0, transpose=True)
        assert so == sg == 0
        assert yg.tobytes() == yo.tobytes()


def test_i64_overflow_and_cast_errors_match():
    rng = np.random.default_rng(2)
    og, gv, *_ = random_graph(rng, 200, 1500, weights="frac")
    x = np.full(200, I64_MAX - 3, np.int64)
    so, _, sg, _ = run_both(og, gv, "plus_times", x, np.zeros(200, np.int64))
    assert so == sg != 0


def test_device_operands_and_async_calls():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    og, gv, *_ = random_graph(rng, 1000, 8000, weights="pos")
    x = values(rng, np.float64, 1000)
    yo = np.zeros(1000)
    O.product(og, 0, x, yo, transpose=True)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(1000, dtype=torch.float64, device="cuda")
    W.spmv(gv, W.Product("plus_times", transpose=True), xd, yd, asynchronous=True)
    gv.sync()
    assert yd.cpu().numpy().tobytes() == yo.tobytes()


# ---------------------------------------------------------------- PageRank

def small():
    return [(0, 0, 1, 1.0), (0, 1, 2, 1.0), (1, 2, 3, 1.0), (1, 0, 3, 5.0), (0, 3, 0, 1.0),
            (1, 4, 4, 2.0), (1, 0, 1, 0.5)]


def upload(og):
    off, tgt, w, _, _, _ = og.csr()
    return W.GraphVersion(off, tgt, w)


def test_pagerank_known_answers():
    # compute/pagerank/tests.rs:78-123 on the device: the same iteration
    # counts and, these rows being short, the same ranks.
    og = O.Graph.from_edges(6, small(), weighted=True, relations=2)
    r = W.pagerank(upload(og), None, W.PageRank(0.85, 1e-6, 100))
    assert r.iterations == 14
    exp = np.array([0.28666944658969795, 0.08535717971974721, 0.10168006797333676,
                    0.3029923348432875, 0.19417475728151729, 0.029126213592413387])
    assert np.abs(r.values - exp).sum() / exp.sum() <= 1e-12
    edges = [e for e in small() if e[1] != 1 and e[2] != 1]
    og = O.Graph.from_edges(6, edges, weighted=True, relations=2)
    gv = upload(og)
    tomb = O.tombstone_words(6, [1])
    r = W.pagerank(gv, tomb, W.PageRank(0.85, 1e-6, 100))
    assert r.iterations == 69 and r.values[1] == 0.0
    r = W.pagerank(gv, tomb, W.PageRank(0.85, 1e-6, 100, seed=np.arange(1, 7, dtype=np.float64)))
    assert r.iterations == 71
    exp = np.array([0.2553952337234808, 0, 0.03237410071942446, 0.28777128327185025,
                    0.3597111808463956, 0.06474820143884892])
    assert np.abs(r.values - exp).sum() / exp.sum() <= 1e-12


def test_pagerank_edge_cases():
    og = O.Graph.from_edges(6, small(), weighted=True, relations=2)
    gv = upload(og)
    r = W.pagerank(gv, None, W.PageRank(max_iter=0))
    assert r.iterations == 0 and np.all(r.values == 1.0 / 6.0)
    assert W.pagerank(gv, None, W.PageRank(tol=None, max_iter=7)).iterations == 7
    assert W.pagerank(gv, None, W.PageRank(tol=float("nan"))).iterations == 1
    g3 = upload(O.Graph.from_edges(3, [(0, 0, 1, 1.0)], weighted=False))
    with pytest.raises(W.api.DivisionByZero):
        W.pagerank(g3, O.tombstone_words(3, [0, 1, 2]), W.PageRank(max_iter=0))
    with pytest.raises(W.api.DivisionByZero):
        W.pagerank(g3, None, W.PageRank(seed=np.array([1.0, -1.0, 0.0])))


@pytest.mark.parametrize("weighted", [False, True])
def test_pagerank_rmat16_matches_the_oracle(weighted):
    g = W.rmat(16, seed=1)
    w = W.edge_weights(g, "uniform") if weighted else None
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w)
    gv = W.GraphVersion(g.offsets, g.targets, w)
    ro, it, delta, thr = O.pagerank(og, 0.85, 1e-10, 100)
    r = W.pagerank(gv, None, W.PageRank(0.85, 1e-10, 100))
    assert r.iterations == it
    assert np.abs(r.values - ro).sum() / np.abs(ro).sum() <= 1e-12
    tomb = O.tombstone_words(g.id_space, range(0, g.id_space, 97))
    seed = np.random.default_rng(1).random(g.id_space)
    ro, it, _, _ = O.pagerank(og, 0.85, 1e-10, 100, tombstones=tomb, seed=seed)
    r = W.pagerank(gv, tomb, W.PageRank(0.85, 1e-10, 100, seed=seed))
    assert r.iterations == it
    assert np.abs(r.values - ro).sum() / np.abs(ro).sum() <= 1e-12


# ---------------------------------------------------------------- traversal

def directed(n, pairs, reverse=True):
    og = O.Graph.from_edges(n, [(0, s, t, 1.0) for s, t in pairs], weighted=False)
    off, tgt, _, _, _, _ = og.csr()
    return og, W.GraphVersion(off, tgt, None, reverse=reverse)


def visits(t):
    return [(v.node, v.depth, v.via) for v in t.result]


def test_bfs_known_answers():
    og, gv = directed(6, [(0, 1), (1, 2), (2, 3), (0, 4), (4, 3), (2, 2)])
    t = W.bfs(gv, [0])
    assert visits(t) == [(0, 0, None), (1, 1, 0), (4, 1, 0), (2, 2, 1), (3, 2, 4)]
    assert (t.stats.nodes_visited, t.stats.edges_traversed, t.stats.truncated) == (5, 6, False)
    assert visits(W.bfs(gv, [2, 4, 2])) == [(2, 0, None), (4, 0, None), (3, 1, 2)]
    assert visits(W.bfs(gv, [4, 1])) == [(4, 0, None), (1, 0, None), (2, 1, 1), (3, 1, 4)]
    assert [(a, b) for a, b, _ in visits(W.bfs(gv, [3], direction="in"))] == \
        [(3, 0), (2, 1), (4, 1), (1, 2), (0, 2)]
    t = W.bfs(gv, [0], limits=W.Limits(max_results=2))
    assert visits(t) == [(0, 0, None), (1, 1, 0)] and t.stats.truncated
    assert [(a, b) for a, b, _ in visits(W.bfs(gv, [0], filter=[1, 2, 3]))] == \
        [(0, 0), (1, 1), (2, 2), (3, 3)]
    with pytest.raises(W.api.NodeOutsideIdSpace):
        W.bfs(gv, [6])


def test_reachable_set_known_answers():
    og, gv = directed(6, [(0, 1), (0, 2), (0, 3), (1, 5), (2, 4), (3, 1)])
    t = W.reachable_set(gv, [0])
    assert t.result == [0, 1, 2, 3, 4, 5]
    assert t.stats.nodes_visited == 6 and t.stats.edges_traversed == 5
    og, gv = directed(6, [(0, 1), (1, 2), (2, 3), (4, 3)])
    assert W.reachable_set(gv, [1, 4]).result == [1, 4, 2, 3]
    assert W.reachable_set(gv, [0], max_depth=1).result == [0, 1]
    assert W.reachable(gv, 0, 3).result and not W.reachable(gv, 0, 3, max_depth=2).result


def compare_bfs(og, gv, starts, **kw):
    ov, ost = O.bfs(og, starts, direction={"out": 0, "in": 1, "both": 2}[kw.get("direction", "out")],
                    max_depth=kw.get("max_depth"), max_results=kw.get("max_results"),
                    filter_ids=kw.get("filter"))
    t = W.bfs(gv, starts, filter=kw.get("filter"), direction=kw.get("direction", "out"),
              limits=W.Limits(kw.get("max_depth"), kw.get("max_results")))
    assert visits(t) == ov
    assert t.stats.nodes_visited == ost["nodes_visited"]
    assert t.stats.edges_traversed == ost["edges_traversed"]
    assert t.stats.truncated == ost["truncated"]


def test_bfs_rmat16_64_seeds_depth_8_bit_exact():
    g = W.rmat(16, seed=1)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    rng = np.random.default_rng(1)
    for s in rng.integers(0, g.id_space, 64):
        compare_bfs(og, gv, [int(s)], max_depth=8)


def test_bfs_directions_filters_truncation_random():
    rng = np.random.default_rng(4)
    for trial in range(25):
        n = int(rng.integers(5, 400))
        pairs = [(int(rng.integers(0, n)), int(rng.integers(0, n))) for _ in range(int(rng.integers(0, 6 * n)))]
        og, gv = directed(n, pairs)
        starts = [int(v) for v in rng.integers(0, n, int(rng.integers(1, 4)))]
        for direction in ("out", "in", "both"):
            filt = [int(v) for v in rng.choice(n, n // 2, replace=False)] if trial % 3 == 0 else None
            depth = None if trial % 2 else int(rng.integers(0, 5))
            results = None if trial % 4 else int(rng.integers(0, n))
            compare_bfs(og, gv, starts, direction=direction, filter=filt, max_depth=depth,
                        max_results=results)
            nodes, st = O.reachable_set(og, starts, direction={"out": 0, "in": 1, "both": 2}[direction],
                                        max_depth=depth)
            t = W.reachable_set(gv, starts, max_depth=depth, direction=direction)
            assert t.result == nodes
            assert t.stats.edges_traversed == st["edges_traversed"]


def test_reachable_set_rmat16_matches_including_pulled_levels():
    g = W.rmat(16, seed=1)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    for s in (0, 17, 4242):
        nodes, st = O.reachable_set(og, [s])
        t = W.reachable_set(gv, [s])
        assert t.result == nodes
        assert t.stats.edges_traversed == st["edges_traversed"]
        assert t.stats.nodes_visited == st["nodes_visited"]
        assert t.stats.pulled_levels == st["pulled_levels"]


def test_components_match_the_oracle():
    # traversal/components.rs: the reference's example, then R-MAT graphs
    # (many components, directed) and a chain whose roots settle late.
    g = O.Graph.from_edges(7, [(0, s, t, 1.0) for s, t in [(4, 2), (2, 0), (3, 1), (5, 1), (6, 6)]],
                           weighted=False)
    off, tgt, _, _, _, _ = g.csr()
    labels, stats = W.components(W.GraphVersion(off, tgt))
    assert list(labels) == [0, 1, 0, 1, 0, 1, 6]
    assert (stats.nodes_visited, stats.edges_traversed) == (7, 5)
    for scale, seed in ((10, 1), (14, 2), (16, 3)):
        hg = W.rmat(scale, seed=seed)
        og = O.Graph.from_csr(hg.id_space, hg.offsets, hg.targets, reverse=False)
        want, nv, ne = O.components(og)
        got, st = W.components(hg.upload())
        assert np.array_equal(got, want)
        assert (st.nodes_visited, st.edges_traversed) == (nv, ne)
    n = 5000
    chain = [(0, i + 1, i, 1.0) for i in range(n - 1)][::-1]
    og = O.Graph.from_edges(n, chain, weighted=False)
    off, tgt, _, _, _, _ = og.csr()
    got, _ = W.components(W.GraphVersion(off, tgt))
    assert np.all(got == 0)


@pytest.mark.parametrize("width", [2, 3, 5, 16, 33])
def test_spmm_hub_rows_every_width(width):
    # Rows far over 256 entries (pieces combined in order) and widths that
    # leave part of a column block idle; values are halves, so every sum is
    # exact whatever the grouping.
    rng = np.random.default_rng(width)
    og, gv, *_ = hub_graph(rng, 6000, 4000)
    n = gv.id_space
    for semiring, dtype in (("plus_times", np.float64), ("min_plus", np.int64),
                            ("max_times", np.float64), ("lor_land", np.uint8)):
        x = values(rng, dtype, n, width=width)
        y0 = values(rng, dtype, n, width=width)
        for transpose in (False, True):
            so, yo, sg, yg = run_both(og, gv, semiring, x, y0, transpose=transpose)
            assert so == sg
            if not so:
                assert yg.tobytes() == yo.tobytes(), (semiring, transpose)
    mask = (rng.random(n) < 0.5).astype(np.float64)
    x = values(rng, np.float64, n, width=width)
    y0 = values(rng, np.float64, n, width=width)
    so, yo, sg, yg = run_both(og, gv, "plus_times", x, y0, mask=mask, complement=True,
                              replace=True, accumulate="plus", transpose=True)
    assert so == sg == 0
    assert yg.tobytes() == yo.tobytes()


def test_bfs_long_and_huge_rows_match_the_oracle():
    # Rows over 2,048 entries go to the long-row push (a block each) and
    # rows over 32,768 to the whole-grid push: two hubs of 40,000 and
    # 5,000 out-edges beside random edges, every direction, seeds that
    # reach the hubs at different levels.
    rng = np.random.default_rng(21)
    n = 50000
    pairs = set()
    for t in rng.choice(n, 40000, replace=False):
        pairs.add((7, int(t)))
    for t in rng.choice(n, 5000, replace=False):
        pairs.add((11, int(t)))
    for _ in range(3 * n):
        pairs.add((int(rng.integers(0, n)), int(rng.integers(0, n))))
    pairs.add((3, 7))
    og, gv = directed(n, sorted(pairs))
    for starts in ([7], [3], [11, 40000], [int(rng.integers(0, n))]):
        for direction in ("out", "in", "both"):
            compare_bfs(og, gv, starts, direction=direction)
            compare_bfs(og, gv, starts, direction=direction, max_depth=2)
