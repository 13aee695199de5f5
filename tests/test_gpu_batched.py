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


def ragged_graph(n, seed):
    """n nodes (not a multiple of 4): a path 1 -> 2 -> ... -> 70 -> 0 that
    nothing else enters (depths past 31), a hub 0 with an edge to every node
    from 71 on (out-degree above 2^16) and 0 to 3 random edges from each of
    those nodes to the others or the hub; targets sorted and distinct per
    row."""
    rng = np.random.default_rng(seed)
    rows = [np.arange(71, n)]
    rows += [np.array([u + 1]) for u in range(1, 70)]
    rows.append(np.array([0]))
    for u in range(71, n):
        t = rng.integers(70, n, rng.integers(0, 4))
        t[t == 70] = 0
        rows.append(np.unique(t[t != u]))
    offsets = np.zeros(n + 1, np.uint32)
    offsets[1:] = np.cumsum([len(r) for r in rows])
    targets = np.concatenate(rows).astype(np.uint32)
    og = O.Graph.from_csr(n, offsets, targets, reverse=False)
    return og, W.GraphVersion(offsets, targets)


@pytest.mark.parametrize("width,cap_hi", [(37, 17), (37, 201), (1030, 201)])
def test_bfs_batched_ragged_sizes_deep_caps_and_a_wide_hub(width, cap_hi):
    # Node count not a multiple of 4 (partial tiles, byte stores), source
    # counts not a multiple of 4, caps above 31 (eight depth bit planes) and
    # a node of out-degree above 2^16 (the plain degree sum).
    n = 70_003
    og, gv = ragged_graph(n, seed=width + cap_hi)
    rng = np.random.default_rng(cap_hi)
    src = rng.integers(0, n, width).astype(np.uint64)
    src[:3] = [0, 1, 5]
    caps = rng.integers(0, cap_hi, width).astype(np.uint32)
    caps[:3] = cap_hi - 1
    d, e = W.bfs_batched(gv, src, caps)
    do, eo = O.bfs_depths(og, src, caps)
    assert np.array_equal(d, do)
    assert np.array_equal(e, eo)


def path_version(n):
    """The path 0 -> 1 -> ... -> n-1."""
    offsets = np.minimum(np.arange(n + 1), n - 1).astype(np.uint64)
    targets = np.arange(1, n).astype(np.uint32)
    return O.Graph.from_csr(n, offsets, targets, reverse=False), W.GraphVersion(offsets, targets)


def test_bfs_batched_caps_above_254_are_served_or_refused_never_cut_short():
    # Depths are bytes (255: not reached), so a pass runs 254 levels at most.
    # traversal/level.rs:119-123 and limits.rs:8: a cap is any u32.  A search
    # that ends within 254 levels is served whatever its cap; one that still
    # expands at depth 254 with a deeper cap is refused (Unsupported), so
    # the adapter keeps the native search, rather than answered with 255s.
    og, gv = path_version(300)
    with pytest.raises(W.Unsupported):
        W.bfs_batched(gv, [0], [300])
    with pytest.raises(W.Unsupported):  # one offending source among many
        src = np.arange(40, dtype=np.uint64) + 10
        caps = np.full(40, 16, np.uint32)
        caps[7] = 1000
        src[7] = 0
        W.bfs_batched(gv, src, caps)
    # Cap 254 from 0 stops at node 254; from 50 and 100 the path ends at
    # depths 249 and 199, below their caps of 300 and 2^32 - 1.
    src = np.array([0, 0, 50, 100], np.uint64)
    caps = np.array([254, 100, 300, 2**32 - 1], np.uint32)
    d, e = W.bfs_batched(gv, src, caps)
    do, eo = O.bfs_depths(og, src, caps)
    assert np.array_equal(d, do) and np.array_equal(e, eo)
    assert d[0, 254] == 254 and d[0, 255] == 255 and d[2, 299] == 249 and d[3, 299] == 199
    og2, gv2 = path_version(200)
    d, e = W.bfs_batched(gv2, [0], [2**32 - 1])
    do, eo = O.bfs_depths(og2, np.array([0], np.uint64), np.array([2**32 - 1], np.uint32))
    assert np.array_equal(d, do) and np.array_equal(e, eo) and d[0, 199] == 199


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


def weighted_graph(scale, kind, seed=1):
    g = W.rmat(scale, seed=seed)
    w = W.edge_weights(g, kind)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w)
    return g, w, og, W.GraphVersion(g.offsets, g.targets, w)


@pytest.mark.parametrize("columns", [1, 4, 32])
def test_minplus_batched_equals_the_sssp_loop_per_source(columns):
    g, w, og, gv = weighted_graph(13, "int")
    rng = np.random.default_rng(columns)
    width = 70
    src = rng.integers(0, g.id_space, width).astype(np.uint64)
    hops = rng.integers(0, 17, width).astype(np.uint32)
    W.set_schedule(gv, "minplus", width, columns)
    d, it = W.minplus_batched(gv, src, hops)
    do, ito = O.sssp_i64(og, src, hops)
    assert np.array_equal(d, do)
    assert np.array_equal(it, ito)


@pytest.mark.parametrize("kind", ["wide", "negative", "fraction"])
def test_minplus_batched_wide_negative_and_fractional_weights(kind):
    # Weights of 2^28 with caps to 16 leave the 32-bit range (the i64 path);
    # negative integer weights and non-integral weights (cast to i64 per
    # edge, round half to even) take their own paths; all equal the loop.
    g = W.rmat(12, seed=9)
    rng = np.random.default_rng(3)
    if kind == "wide":
        w = rng.integers(1, 4, g.edges).astype(np.float64) * 2.0 ** 28
    elif kind == "negative":
        w = rng.integers(-3, 100, g.edges).astype(np.float64)
    else:
        w = rng.integers(0, 400, g.edges) / 4.0
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w)
    gv = W.GraphVersion(g.offsets, g.targets, w)
    src = rng.integers(0, g.id_space, 50).astype(np.uint64)
    hops = rng.integers(0, 17, 50).astype(np.uint32)
    d, it = W.minplus_batched(gv, src, hops)
    do, ito = O.sssp_i64(og, src, hops)
    assert np.array_equal(d, do)
    assert np.array_equal(it, ito)


def test_minplus_batched_unweighted_and_capped():
    g = W.rmat(12, seed=4)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    src = np.arange(40, dtype=np.uint64) * 13
    hops = np.array([0, 1, 2, 3, 16] * 8, np.uint32)
    d, it = W.minplus_batched(gv, src, hops)
    do, ito = O.sssp_i64(og, src, hops)
    assert np.array_equal(d, do) and np.array_equal(it, ito)


@pytest.mark.parametrize("weighted", [False, True])
def test_ppr_batched_matches_seeded_pagerank_per_column(weighted):
    g = W.rmat(14, seed=2)
    w = W.edge_weights(g, "uniform") if weighted else None
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w)
    gv = W.GraphVersion(g.offsets, g.targets, w)
    rng = np.random.default_rng(7)
    sets = [rng.choice(g.id_space, int(np.exp(rng.uniform(0, np.log(300)))), replace=False)
            for _ in range(19)]
    W.set_schedule(gv, "ppr", len(sets), 8 if weighted else 2)
    r, it = W.ppr_batched(gv, sets, W.PageRank(0.85, 1e-10, 100))
    for c, s in enumerate(sets):
        seed = np.zeros(g.id_space)
        seed[s] = 1.0
        ro, ito, _, _ = O.pagerank(og, 0.85, 1e-10, 100, seed=seed)
        assert it[c] == ito
        assert np.abs(r[c] - ro).sum() / np.abs(ro).sum() <= 1e-12


@pytest.mark.parametrize("slots,count,tol,max_iter", [
    (32, 3, 1e-10, 100),   # fewer sets than slots
    (8, 70, 1e-10, 100),   # every slot refilled many times
    (16, 40, None, 7),     # no tolerance: every set stops at max_iter together
    (8, 12, 1e-6, 3),      # max_iter cuts some sets, the tolerance others
    (32, 5, 1e-10, 0),     # no iteration: the start vector
])
def test_ppr_batched_slots_refill_in_any_order(slots, count, tol, max_iter):
    # A slot whose set stops takes the next set; each set's ranks and
    # iteration count must still be its own plain seeded PageRank's, and a
    # second call (the captured chunk replayed) must repeat them.
    g = W.rmat(13, seed=9)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    rng = np.random.default_rng(count)
    sets = [rng.integers(0, g.id_space, int(np.exp(rng.uniform(0, np.log(200))))) for _ in range(count)]
    sets[0] = np.concatenate([sets[0], sets[0][:1]])  # a repeated node counts once
    W.set_schedule(gv, "ppr", count, slots, 3)
    pr = W.PageRank(0.85, tol, max_iter)
    r, it = W.ppr_batched(gv, sets, pr)
    r2, it2 = W.ppr_batched(gv, sets, pr)
    assert np.array_equal(it, it2) and r.tobytes() == r2.tobytes()
    for c, s in enumerate(sets):
        seed = np.zeros(g.id_space)
        seed[s] = 1.0
        ro, ito, _, _ = O.pagerank(og, 0.85, tol, max_iter, seed=seed)
        assert it[c] == ito, c
        assert np.abs(r[c] - ro).sum() / np.abs(ro).sum() <= 1e-12, c


def test_autotuners_pick_valid_schedules():
    g, w, og, gv = weighted_graph(12, "int")
    s = W.autotune(gv, "minplus", 100)
    assert s.columns_per_pass in (4, 8, 16, 32)
    s = W.autotune(gv, "ppr", 100)
    assert s.columns_per_pass in (8, 16, 32)


@pytest.mark.parametrize("count", [1, 8, 600])
def test_bfs_batched_push_and_pull_levels_agree(count):
    # Few sources keep the early frontiers under the push threshold (the
    # levels scatter over the forward CSR); many reach the pull levels.  A
    # graph with hubs and a repeated call check the accumulators are left
    # clear between levels and calls.
    g, og, gv = graph(13, seed=4)
    rng = np.random.default_rng(count)
    src = rng.integers(0, g.id_space, count).astype(np.uint64)
    caps = rng.integers(1, 17, count).astype(np.uint32)
    do, eo = O.bfs_depths(og, src, caps)
    for _ in range(2):
        d, e = W.bfs_batched(gv, src, caps)
        assert np.array_equal(d, do)
        assert np.array_equal(e, eo)


def test_bfs_batched_after_other_calls_on_the_version():
    # Scratch that the batched search keeps zero between calls is not
    # shared with other calls' scratch (top_k, the batched searches of
    # other kinds).
    g, og, gv = graph(12, seed=6)
    rng = np.random.default_rng(8)
    src = rng.integers(0, g.id_space, 200).astype(np.uint64)
    caps = rng.integers(1, 17, 200).astype(np.uint32)
    do, eo = O.bfs_depths(og, src, caps)
    W.bfs_batched(gv, src, caps)
    W.top_k(gv, rng.random(g.id_space), 50)
    W.minplus_batched(gv, src[:40], caps[:40])
    d, e = W.bfs_batched(gv, src, caps)
    assert np.array_equal(d, do)
    assert np.array_equal(e, eo)
