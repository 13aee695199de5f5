"""The oracle against the reference's own known-answer tests.

Every expected value below is copied from a test in the reference's source
tree (path within the reference project, file:line).  These pin the C++
restatement before it is trusted as the checker of the CUDA kernels.
"""

import math
import struct

import numpy as np
import pytest

import oracle as O

F32, F64, I64, BOOL = 0, 1, 2, 3
FIRST, SECOND, PAIR, PLUS, TIMES, MIN, MAX, LOR, LAND, ANY = range(10)
PLUS_TIMES, MIN_PLUS, MAX_PLUS, MAX_TIMES, MIN_TIMES, LOR_LAND = 0, 1, 2, 3, 4, 5
PLUS_FIRST = 8

# status codes (include/warren_cuda.h)
BIGINT, FLOAT_OVER, FLOAT_UNDER, DIV0 = 10, 11, 12, 13
NODE_OUTSIDE = 20

NAN, INF = float("nan"), float("inf")
I64_MAX, I64_MIN = 2**63 - 1, -(2**63)


def _pack(dtype, v):
    if dtype == F64:
        return np.array([v], np.float64)
    if dtype == F32:
        return np.array([v], np.float32)
    if dtype == I64:
        return np.array([v], np.int64)
    return np.array([1 if v else 0], np.uint8)


def apply(dtype, op, a, b):
    a, b = _pack(dtype, a), _pack(dtype, b)
    out = _pack(dtype, 0)
    st = O.lib().wo_apply(dtype, op, a.ctypes.data, b.ctypes.data, out.ctypes.data)
    return st, out[0]


def mult(dtype, add, mul, w, v):
    w, v = _pack(dtype, w), _pack(dtype, v)
    out = _pack(dtype, 0)
    st = O.lib().wo_multiply(dtype, add, mul, w.ctypes.data, v.ctypes.data, out.ctypes.data)
    return st, out[0]


def from_weight(dtype, w):
    out = _pack(dtype, 0)
    st = O.lib().wo_from_weight(dtype, w, out.ctypes.data)
    return st, out[0]


def table(dtype, a, b):
    rows = [apply(dtype, op, a, b) for op in range(10)]
    assert all(st == 0 for st, _ in rows)
    return [v for _, v in rows]


def test_semiring_add_and_multiply_by_name(oracle):
    # compute/semiring.rs:410-422: each semiring is <add>_<mult>.
    names = ["plus_times", "min_plus", "max_plus", "max_times", "min_times", "lor_land",
             "any_pair", "plus_pair", "plus_first", "plus_second", "min_first", "min_second",
             "max_second"]
    ops = ["first", "second", "pair", "plus", "times", "min", "max", "lor", "land", "any"]
    for s, name in enumerate(names):
        add, mul = name.split("_")
        assert ops[O.lib().wo_semiring_add(s)] == add
        assert ops[O.lib().wo_semiring_mul(s)] == mul


def test_identities_are_the_no_entry_values(oracle):
    # compute/semiring.rs:437-445
    monoids = [PLUS, MIN, MAX, LOR, ANY]
    def ident(dtype):
        out = []
        for m in monoids:
            o = _pack(dtype, 0)
            O.lib().wo_identity(dtype, m, o.ctypes.data)
            out.append(o[0])
        return out
    assert ident(F64) == [0.0, INF, -INF, 0.0, 0.0]
    assert ident(F32) == [0.0, INF, -INF, 0.0, 0.0]
    assert ident(I64) == [0, I64_MAX, I64_MIN, 0, 0]
    assert ident(BOOL) == [0, 1, 0, 0, 0]


def test_binary_ops_on_each_element_type(oracle):
    # compute/semiring.rs:451-461
    assert table(F64, 2.0, -3.0) == [2.0, -3.0, 1.0, -1.0, -6.0, -3.0, 2.0, 1.0, 1.0, 2.0]
    assert table(F32, 0.0, 4.0) == [0.0, 4.0, 1.0, 4.0, 0.0, 0.0, 4.0, 1.0, 0.0, 0.0]
    assert table(I64, 5, 0) == [5, 0, 1, 5, 0, 0, 5, 1, 0, 5]
    assert table(BOOL, 1, 0) == [1, 0, 1, 1, 0, 0, 1, 1, 0, 1]


def test_min_and_max_order_nan_above_every_number(oracle):
    # compute/semiring.rs:463-472
    assert apply(F64, MIN, NAN, 1.0) == (0, 1.0)
    assert math.isnan(apply(F64, MAX, 1.0, NAN)[1])
    assert apply(F64, MIN, INF, NAN) == (0, INF)
    assert apply(F64, LOR, NAN, 0.0) == (0, 1.0)
    st, v = apply(F64, MIN, -0.0, 0.0)
    assert math.copysign(1.0, v) < 0


def test_i64_identities_absorb_plus(oracle):
    # compute/semiring.rs:474-489
    assert mult(I64, MIN, PLUS, 3, I64_MAX) == (0, I64_MAX)
    assert mult(I64, MIN, PLUS, -3, I64_MAX) == (0, I64_MAX)
    assert mult(I64, MAX, PLUS, 3, I64_MIN) == (0, I64_MIN)
    assert mult(I64, MIN, PLUS, 3, 4) == (0, 7)
    assert mult(I64, MIN, PLUS, 1, I64_MAX - 1) == (0, I64_MAX)
    assert mult(I64, MIN, PLUS, 2, I64_MAX - 1)[0] == BIGINT
    assert mult(I64, MAX, PLUS, 1, I64_MAX)[0] == BIGINT
    assert mult(F64, MIN, PLUS, 1.0, INF) == (0, INF)


def test_i64_identities_absorb_times_by_a_positive_weight(oracle):
    # compute/semiring.rs:491-508
    assert mult(I64, MIN, TIMES, 3, I64_MAX) == (0, I64_MAX)
    assert mult(I64, MAX, TIMES, 3, I64_MIN) == (0, I64_MIN)
    assert mult(I64, MIN, TIMES, 1, I64_MAX) == (0, I64_MAX)
    assert mult(I64, MIN, TIMES, 0, I64_MAX) == (0, 0)
    assert mult(I64, MIN, TIMES, -1, I64_MAX) == (0, -I64_MAX)
    assert mult(I64, MIN, TIMES, -2, I64_MAX)[0] == BIGINT
    assert mult(I64, MAX, TIMES, -1, I64_MIN)[0] == BIGINT
    assert mult(I64, MIN, TIMES, 2, I64_MAX // 2 + 1)[0] == BIGINT
    assert mult(I64, MAX, TIMES, 2, I64_MAX)[0] == BIGINT


def test_i64_overflow_is_an_error(oracle):
    # compute/semiring.rs:510-517
    assert apply(I64, PLUS, I64_MAX, 1)[0] == BIGINT
    assert apply(I64, TIMES, I64_MIN, -1)[0] == BIGINT


def test_weights_convert_as_sql_casts(oracle):
    # compute/semiring.rs:519-533
    assert from_weight(F64, 0.1) == (0, 0.1)
    assert from_weight(F32, 0.1) == (0, np.float32(0.1))
    assert from_weight(F32, 1e300)[0] == FLOAT_OVER
    assert from_weight(F32, 1e-300)[0] == FLOAT_UNDER
    assert from_weight(F32, INF) == (0, np.float32(INF))
    assert from_weight(I64, 2.5) == (0, 2)
    assert from_weight(I64, 3.5) == (0, 4)
    assert from_weight(I64, -2.5) == (0, -2)
    assert from_weight(I64, 9.3e18)[0] == BIGINT
    assert from_weight(I64, NAN)[0] == BIGINT
    assert from_weight(BOOL, 0.0) == (0, 0)
    assert from_weight(BOOL, NAN) == (0, 1)


def _same(found, expected):
    st, v = found
    if isinstance(expected, int):
        assert st == expected
        return
    assert st == 0
    if math.isnan(expected):
        assert math.isnan(v)
    else:
        assert struct.pack("<d", v) == struct.pack("<d", expected), (v, expected)


def test_float_operators_check_like_float_c(oracle):
    # compute/map/arithmetic.rs:237-258 (f64 rows)
    A, S, M, D = 0, 1, 2, 3
    _same(O.float_op(D, NAN, 0.0), NAN)
    _same(O.float_op(D, 1.0, 0.0), DIV0)
    _same(O.float_op(D, 0.0, -0.0), DIV0)
    _same(O.float_op(D, INF, 0.0), DIV0)
    _same(O.float_op(M, 1e308, 10.0), FLOAT_OVER)
    _same(O.float_op(M, 1e-308, 1e-10), 1e-318)
    _same(O.float_op(M, 1e-308, 1e-100), FLOAT_UNDER)
    _same(O.float_op(M, INF, 0.0), NAN)
    _same(O.float_op(S, INF, INF), NAN)
    _same(O.float_op(A, 1e308, 1e308), FLOAT_OVER)
    _same(O.float_op(A, INF, 1.0), INF)
    _same(O.float_op(D, 1.0, 1e-310), FLOAT_OVER)
    _same(O.float_op(D, 1e-320, 1e10), FLOAT_UNDER)
    _same(O.float_op(D, 1.0, INF), 0.0)
    _same(O.float_op(D, INF, INF), NAN)
    _same(O.float_op(M, -0.0, 1.0), -0.0)


# ---------------------------------------------------------------- PageRank

def small():
    # compute/pagerank/tests.rs:53-66: nodes 1-6 as dense ids 0-5, relations
    # a (0) and b (1), weighted; node 6 has no edge.
    return [(0, 0, 1, 1.0), (0, 1, 2, 1.0), (1, 2, 3, 1.0), (1, 0, 3, 5.0), (0, 3, 0, 1.0),
            (1, 4, 4, 2.0), (1, 0, 1, 0.5)]


@pytest.mark.parametrize("chunk", [4, 65536])
def test_pagerank_ranks_are_those_the_plpgsql_library_wrote(oracle, chunk):
    # compute/pagerank/tests.rs:78-123: exact ranks, 14 / 69 / 71 iterations.
    O.set_chunk(chunk)
    try:
        g = O.Graph.from_edges(6, small(), weighted=True, relations=2)
        ranks, it, _, _ = O.pagerank(g, 0.85, 1e-6, 100)
        assert it == 14
        assert list(ranks) == [0.28666944658969795, 0.08535717971974721, 0.10168006797333676,
                               0.3029923348432875, 0.19417475728151729, 0.029126213592413387]

        edges = [e for e in small() if e[1] != 1 and e[2] != 1]
        g = O.Graph.from_edges(6, edges, weighted=True, relations=2)
        tomb = O.tombstone_words(6, [1])
        ranks, it, _, _ = O.pagerank(g, 0.85, 1e-6, 100, tombstones=tomb)
        assert it == 69
        live = [(i + 1, ranks[i]) for i in range(6) if i != 1]
        assert live == [(1, 0.33506897700306837), (3, 0.03614457831325302),
                        (4, 0.3516780109487391), (5, 0.24096385542168675),
                        (6, 0.03614457831325302)]
        assert ranks[1] == 0.0

        seed = np.arange(1, 7, dtype=np.float64)
        ranks, it, _, _ = O.pagerank(g, 0.85, 1e-6, 100, tombstones=tomb, seed=seed)
        assert it == 71
        live = [(i + 1, ranks[i]) for i in range(6) if i != 1]
        assert live == [(1, 0.2553952337234808), (3, 0.03237410071942446),
                        (4, 0.28777128327185025), (5, 0.3597111808463956),
                        (6, 0.06474820143884892)]
    finally:
        O.set_chunk(65536)


def test_pagerank_ring_and_seed(oracle):
    # compute/pagerank/tests.rs:125-137
    g = O.Graph.from_edges(4, [(0, n, (n + 1) % 4, 1.0) for n in range(4)], weighted=False)
    ranks, _, _, _ = O.pagerank(g, 0.85, 1e-12, 100)
    assert all(abs(r - 0.25) < 1e-12 for r in ranks)
    ranks, _, _, _ = O.pagerank(g, 0.85, 1e-12, 100, seed=np.array([1.0, 0, 0, 0]))
    assert abs(ranks.sum() - 1.0) < 1e-12
    assert ranks[0] > ranks[1] > ranks[2] > ranks[3]


def test_pagerank_no_iterations_and_no_tol(oracle):
    # compute/pagerank/tests.rs:139-153
    g = O.Graph.from_edges(6, small(), weighted=True, relations=2)
    ranks, it, _, _ = O.pagerank(g, 0.85, 1e-6, 0)
    assert it == 0 and list(ranks) == [1.0 / 6.0] * 6
    _, it, _, _ = O.pagerank(g, 0.85, None, 7)
    assert it == 7
    _, it, _, _ = O.pagerank(g, 0.85, NAN, 100)
    assert it == 1


def test_pagerank_refuses_what_cannot_be_divided(oracle):
    # compute/pagerank/tests.rs:155-169
    g = O.Graph.from_edges(3, [(0, 0, 1, 1.0)], weighted=False)
    with pytest.raises(O.OracleError) as e:
        O.pagerank(g, 0.85, 1e-6, 0, tombstones=O.tombstone_words(3, [0, 1, 2]))
    assert e.value.status == DIV0
    with pytest.raises(O.OracleError) as e:
        O.pagerank(g, 0.85, 1e-6, 100, seed=np.array([1.0, -1.0, 0.0]))
    assert e.value.status == DIV0


# ---------------------------------------------------------------- products

def test_i64_min_plus_supersteps_keep_unreached_nodes_at_the_identity(oracle):
    # compute/product/tests.rs:160-186
    g = O.Graph.from_edges(3, [(0, 0, 1, 1.0), (0, 2, 1, 1.0)], weighted=True)
    dist = np.array([0, I64_MAX, I64_MAX], np.int64)
    for _ in range(2):
        x = dist.copy()
        assert O.product(g, MIN_PLUS, x, dist, transpose=True, accumulate=MIN) == 0
        assert list(dist) == [0, 1, I64_MAX]
    y = np.array([I64_MIN] * 3, np.int64)
    assert O.product(g, MAX_PLUS, np.array([5, I64_MIN, I64_MIN], np.int64), y, transpose=True,
                     accumulate=MAX) == 0
    assert list(y) == [I64_MIN, 6, I64_MIN]


def test_i64_min_times_and_max_times_supersteps(oracle):
    # compute/product/tests.rs:486-510
    g = O.Graph.from_edges(3, [(0, 0, 1, 2.0), (0, 2, 1, 3.0)], weighted=True)
    for semiring, acc, ident in [(MIN_TIMES, MIN, I64_MAX), (MAX_TIMES, MAX, I64_MIN)]:
        x = np.array([5, ident, ident], np.int64)
        for _ in range(2):
            inp = x.copy()
            assert O.product(g, semiring, inp, x, transpose=True, accumulate=acc) == 0
            assert x[2] == ident
        assert list(x[:2]) == [5, 10]


def test_i64_plus_times_overflow_is_an_error(oracle):
    # compute/product/tests.rs (i64_overflow_is_an_error)
    g = O.Graph.from_edges(4, [(0, 0, 1, 1.0), (0, 0, 2, 1.0), (0, 1, 3, 1.0)], weighted=False)
    x = np.array([I64_MAX] * 4, np.int64)
    y = np.zeros(4, np.int64)
    assert O.product(g, PLUS_TIMES, x, y) == BIGINT


def test_push_equals_pull_bit_for_bit(oracle):
    # compute/product/tests.rs:447: the push and pull forms agree to the bit.
    rng = np.random.default_rng(3)
    for trial in range(20):
        n = int(rng.integers(1, 40))
        m = int(rng.integers(0, 4 * n + 1))
        edges = [(int(rng.integers(0, 2)), int(rng.integers(0, n)), int(rng.integers(0, n)),
                  float(rng.choice([0.1, 0.7, 1e-3, 3.0, -0.0]))) for _ in range(m)]
        g = O.Graph.from_edges(n, edges, weighted=True, relations=2)
        for semiring in range(13):
            for dtype in (np.float64, np.int64, np.uint8):
                x = (rng.standard_normal(n) * 4).astype(dtype)
                y1 = np.zeros(n, dtype)
                y2 = np.zeros(n, dtype)
                s1 = O.product(g, semiring, x, y1, transpose=True)
                s2 = O.product(g, semiring, x, y2, transpose=True, force_push=True)
                assert s1 == s2
                if s1 == 0:
                    assert y1.tobytes() == y2.tobytes()


def test_product_matches_a_dense_naive_reference(oracle):
    # compute/reference.rs:112-157: for each row, ⊕ over ascending columns,
    # then the mask / replace / accumulate write.
    rng = np.random.default_rng(5)
    for trial in range(30):
        n = int(rng.integers(1, 12))
        edges = [(0, int(rng.integers(0, n)), int(rng.integers(0, n)),
                  float(rng.integers(-3, 4))) for _ in range(int(rng.integers(0, 3 * n)))]
        g = O.Graph.from_edges(n, edges, weighted=True)
        a = [[None] * n for _ in range(n)]
        for _, s, t, w in edges:
            a[s][t] = w if a[s][t] is None else a[s][t] + w
        x = rng.integers(-5, 6, n).astype(np.float64)
        mask = (rng.integers(0, 2, n)).astype(np.float64)
        y0 = rng.integers(-5, 6, n).astype(np.float64)
        for transpose in (False, True):
            for replace in (False, True):
                for acc in (-1, PLUS):
                    y = y0.copy()
                    assert O.product(g, PLUS_TIMES, x, y, transpose=transpose, mask=mask,
                                     replace=replace, accumulate=acc) == 0
                    exp = y0.copy()
                    for i in range(n):
                        t = None
                        for j in range(n):
                            e = a[j][i] if transpose else a[i][j]
                            if e is None:
                                continue
                            p = e * x[j]
                            t = p if t is None else t + p
                        if mask[i] == 0:
                            if replace:
                                exp[i] = 0.0
                            continue
                        if acc == -1:
                            exp[i] = 0.0 if t is None else t
                        elif t is not None:
                            exp[i] = exp[i] + t
                    assert y.tobytes() == exp.tobytes()


# ---------------------------------------------------------------- traversal

def directed(n, pairs):
    return O.Graph.from_edges(n, [(0, s, t, 1.0) for s, t in pairs], weighted=False)


def example_bfs():
    # traversal/bfs.rs:123-126: 0 → 1 → 2 → 3, 0 → 4 → 3, 2 → 2, 5 isolated
    return directed(6, [(0, 1), (1, 2), (2, 3), (0, 4), (4, 3), (2, 2)])


def test_bfs_reports_each_reached_node_once_at_its_shortest_depth(oracle):
    # traversal/bfs.rs:143-160
    v, st = O.bfs(example_bfs(), [0])
    assert v == [(0, 0, None), (1, 1, 0), (4, 1, 0), (2, 2, 1), (3, 2, 4)]
    assert (st["nodes_visited"], st["edges_traversed"], st["truncated"]) == (5, 6, False)


def test_bfs_starts_levels_direction_depth_results_filter(oracle):
    g = example_bfs()
    # bfs.rs:162-166
    assert O.bfs(g, [2, 4, 2])[0] == [(2, 0, None), (4, 0, None), (3, 1, 2)]
    # bfs.rs:168-175
    assert O.bfs(g, [4, 1])[0] == [(4, 0, None), (1, 0, None), (2, 1, 1), (3, 1, 4)]
    # bfs.rs:177-182
    assert [(a, b) for a, b, _ in O.bfs(g, [3], direction=1)[0]] == \
        [(3, 0), (2, 1), (4, 1), (1, 2), (0, 2)]
    # bfs.rs:184-193
    v, st = O.bfs(g, [0], max_depth=1)
    assert len(v) == 3 and not st["truncated"]
    assert O.bfs(g, [0], max_depth=0)[0] == [(0, 0, None)]
    # bfs.rs:195-209
    v, st = O.bfs(g, [0], max_results=2)
    assert v == [(0, 0, None), (1, 1, 0)] and st["truncated"]
    v, st = O.bfs(g, [0], max_results=5)
    assert len(v) == 5 and not st["truncated"]
    # bfs.rs:211-218
    v, _ = O.bfs(g, [0], filter_ids=[1, 2, 3])
    assert [(a, b) for a, b, _ in v] == [(0, 0), (1, 1), (2, 2), (3, 3)]
    # bfs.rs:229-235
    with pytest.raises(O.OracleError) as e:
        O.bfs(g, [6])
    assert e.value.status == NODE_OUTSIDE


def test_reachable_set_pulls_a_wide_level_in_ascending_dense_id_order(oracle):
    # traversal/reachable.rs:158-176
    wide = [(0, 1), (0, 2), (0, 3), (1, 5), (2, 4), (3, 1)]
    g = directed(6, wide)
    nodes, st = O.reachable_set(g, [0])
    assert nodes == [0, 1, 2, 3, 4, 5]
    assert st["nodes_visited"] == 6 and st["edges_traversed"] == 5
    assert O.bfs(g, [0])[1]["edges_traversed"] == 6
    assert [a for a, _, _ in O.bfs(g, [0])[0]] == [0, 1, 2, 3, 5, 4]


def test_reachable_set_holds_the_starts_and_everything_they_reach(oracle):
    # traversal/reachable.rs:184-193, 228-236
    g = directed(6, [(0, 1), (0, 2), (0, 3), (4, 5), (5, 4)])
    pulled = O.reachable_set(g, [0])[1]["edges_traversed"]
    pushed = O.bfs(g, [0])[1]["edges_traversed"]
    assert pulled <= pushed
    g = directed(6, [(0, 1), (1, 2), (2, 3), (4, 3)])
    assert O.reachable_set(g, [1, 4])[0] == [1, 4, 2, 3]
    assert O.reachable_set(g, [0], max_depth=1)[0] == [0, 1]
    assert O.reachable_set(g, [])[0] == []


def test_reachable_set_pulls_in_dense_id_order_at_scale(oracle):
    # traversal/reachable.rs:195-218: depth 2 is pulled, in dense id order.
    edges = []
    for i in range(1, 12001):
        edges += [(0, i), (i, 24001 - i), (i, 0)]
    g = directed(1 << 18, edges)
    nodes, _ = O.reachable_set(g, [0])
    assert len(nodes) == 24001
    assert nodes[12001] == 12001


def test_bfs_matches_scipy_breadth_first_depths(oracle):
    # A secondary oracle: scipy's BFS depths on random graphs.
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import shortest_path
    rng = np.random.default_rng(11)
    for trial in range(10):
        n = int(rng.integers(2, 60))
        m = int(rng.integers(0, 4 * n))
        pairs = [(int(rng.integers(0, n)), int(rng.integers(0, n))) for _ in range(m)]
        g = directed(n, pairs)
        start = int(rng.integers(0, n))
        v, _ = O.bfs(g, [start])
        mat = csr_matrix((np.ones(len(pairs)), ([p[0] for p in pairs], [p[1] for p in pairs])),
                         shape=(n, n))
        mat.data[:] = 1
        d = shortest_path(mat, unweighted=True, indices=start)
        exp = {i: int(d[i]) for i in range(n) if np.isfinite(d[i])}
        assert {a: b for a, b, _ in v} == exp
        nodes, _ = O.reachable_set(g, [start])
        assert sorted(nodes) == sorted(exp)


# ---------------------------------------------------------------- random

def test_uniform_values_depend_only_on_seed_stream_and_node(oracle):
    # compute/random.rs:31-46
    u = O.uniform
    assert u(7, 0, 3) == u(7, 0, 3)
    assert u(7, 0, 3) != u(8, 0, 3)
    assert u(7, 0, 3) != u(7, 1, 3)
    assert u(7, 0, 3) != u(7, 0, 4)
    vals = [u(1, 0, i) for i in range(10000)]
    assert all(-1.0 <= v < 1.0 for v in vals)
    assert abs(sum(vals) / len(vals)) < 0.05
    assert min(vals) < -0.9 and max(vals) > 0.9


def test_topk_sql_order_ties_to_smaller_id(oracle):
    # compute/ranking.rs:15-52
    x = np.array([1.0, 3.0, NAN, 3.0, -1.0])
    nodes, vals = O.topk(x, 3, descending=True)
    assert list(nodes) == [2, 1, 3]
    nodes, vals = O.topk(x, 2, descending=False)
    assert list(nodes) == [4, 0]
    nodes, _ = O.topk(x, 10, descending=True, tombstones=O.tombstone_words(5, [2]))
    assert list(nodes) == [1, 3, 0, 4]


def test_components_label_by_smallest_dense_id(oracle):
    # traversal/components.rs:64-77: {0, 2, 4} via 4 → 2 → 0, {1, 3, 5} via
    # 3 → 1 and 5 → 1, 6 alone; 7 nodes visited, 5 edges traversed.
    g = directed(7, [(4, 2), (2, 0), (3, 1), (5, 1), (6, 6)])
    labels, nodes, edges = O.components(g)
    assert list(labels) == [0, 1, 0, 1, 0, 1, 6]
    assert (nodes, edges) == (7, 5)


def centrality_example():
    # compute/centrality/tests.rs:117-124, with its self-loop.
    return directed(5, [(0, 1), (1, 2), (2, 3), (0, 2), (3, 0), (1, 3), (4, 1), (2, 2)])


def test_closeness_and_harmonic_use_incoming_distances(oracle):
    # compute/centrality/tests.rs:117-143 (NetworkX's values).
    g = centrality_example()
    every = O.sample_sources(5)
    for wf in (True, False):
        assert np.allclose(O.centrality(g, "closeness", every, wf_improved=wf),
                           [0.5, 4 / 7, 2 / 3, 2 / 3, 0.0], rtol=1e-15, atol=0)
    assert np.allclose(O.centrality(g, "harmonic", every), [7 / 3, 17 / 6, 3, 3, 0],
                       rtol=1e-15, atol=0)
    two = O.sample_sources(5, population=np.array([1, 0, 1, 0, 0]))
    assert list(two) == [0, 2]
    assert np.allclose(O.centrality(g, "harmonic", two),
                       [0.5 * 4, 4 / 3 * 2, 1 * 4, 1.5 * 2, 0], rtol=1e-15, atol=0)


def test_source_sampling_known_answers(oracle):
    # compute/centrality/sources.rs:150-190.
    import pg_warren_b200 as W
    tomb = W.node_set(5, [2])
    assert list(O.sample_sources(5, tombstones=tomb)) == [0, 1, 3, 4]
    sel = np.array([1, 0, 1, 1, 0])
    assert list(O.sample_sources(5, tombstones=W.node_set(5, [3]), population=sel)) == [0, 2]
    assert list(O.sample_sources(4, k=9, seed=3)) == [0, 1, 2, 3]
    a, b = O.sample_sources(1000, k=10, seed=7), O.sample_sources(1000, k=10, seed=8)
    assert list(a) == list(O.sample_sources(1000, k=10, seed=7)) and list(a) != list(b)
    counts = np.zeros(20, int)
    for seed in range(2000):
        counts[O.sample_sources(20, k=5, seed=seed)] += 1
    assert ((400 <= counts) & (counts < 600)).all()


def test_library_sampler_is_the_oracles(oracle):
    # wc_sample_sources is host code: it runs without a device.
    import pg_warren_b200 as W
    rng = np.random.default_rng(3)
    for _ in range(40):
        n = int(rng.integers(1, 300))
        tomb = W.node_set(n, rng.integers(0, n, int(rng.integers(0, 10))))
        pop = rng.integers(0, 2, n) if rng.random() < 0.5 else None
        comp = bool(rng.random() < 0.3)
        k = None if rng.random() < 0.2 else int(rng.integers(0, n + 5))
        seed = int(rng.integers(0, 2**63))
        s = W.Sampling(k=k, seed=seed, population=pop, complement=comp)
        got = W.sample_sources(n, s, tomb)
        want = O.sample_sources(n, tombstones=tomb, population=pop, complement=comp, k=k, seed=seed)
        assert np.array_equal(got, want)


def test_reductions_known_answers(oracle):
    # compute/reduce.rs:326-383.
    x = np.array([3.0, -4.0, 0.0, 1.0])
    found = [O.reduce(x, r, width=2) for r in ("sum", "max", "min", "l1", "l2", "nnz")]
    assert found == [0.0, 3.0, -4.0, 8.0, 26 ** 0.5, 3.0]
    assert O.reduce(np.array([2, -5, 7], np.int64), "sum") == 4.0
    assert O.reduce(np.array([True, False, True]), "sum") == 2.0
    assert O.reduce(np.array([True, False, True]), "nnz") == 2.0
    assert O.reduce(np.array([1.5, -0.5], np.float32), "min") == -0.5
    nan = np.array([1.0, np.nan, -2.0])
    assert np.isnan(O.reduce(nan, "max")) and O.reduce(nan, "min") == -2.0
    assert O.reduce(nan, "nnz") == 3.0 and np.isnan(O.reduce(nan, "sum"))
    empty = np.zeros(0)
    assert O.reduce(empty, "max") is None and O.reduce(empty, "min") is None
    assert (O.reduce(empty, "sum"), O.reduce(empty, "l2"), O.reduce(empty, "nnz")) == (0.0, 0.0, 0.0)
    import pg_warren_b200 as W
    x = np.array([3.0, -4.0, 0.0, -9.0, 1.0, 5.0])
    tomb = W.node_set(3, [1])
    found = [O.reduce(x, r, width=2, tombstones=tomb) for r in ("sum", "max", "min", "l1", "l2", "nnz")]
    assert found == [5.0, 5.0, -4.0, 13.0, 51 ** 0.5, 4.0]
    assert O.reduce(x, "min", width=2, tombstones=W.node_set(3, [0, 1, 2])) is None


def test_norm_diff_known_answers(oracle):
    # compute/reduce.rs:385-395.
    old, new = np.array([1.0, 2.0]), np.array([1.0, 5.0, -4.0])
    assert O.norm_diff(new, old, "l1") == 7.0
    assert O.norm_diff(old, new, "l2") == 5.0
    assert O.norm_diff(old, new, "linf") == 4.0
    assert O.norm_diff(np.array([1, 2], np.int64), old, "l1") == 0.0
    assert O.norm_diff(np.zeros(0), np.zeros(0), "linf") == 0.0


def test_chunked_sums_follow_the_chunk_order(oracle):
    # Over several 65,536-element chunks the result is the chunk partials
    # summed in order, each an in-order sum from +0 (reduce.rs:195-268).
    rng = np.random.default_rng(4)
    x = rng.standard_normal(200_003) * 10.0 ** rng.integers(-8, 9, 200_003)
    parts = []
    for c0 in range(0, len(x), 1 << 16):
        s = 0.0
        for v in x[c0:c0 + (1 << 16)]:
            s = s + float(v)
        parts.append(s)
    total = 0.0
    for p in parts:
        total = total + p
    assert O.reduce(x, "sum") == total


BETWEENNESS_KATS = [  # compute/centrality/tests.rs:86-113 (NetworkX's values)
    (True, True, [0.45, 0.325, 0.325, 0.45, 0.0], [0.625, 0.3125, 0.5625, 0.5, 0.0]),
    (True, False, [0.25, 1 / 24, 1 / 24, 0.25, 0.0], [1 / 3, 1 / 12, 1 / 6, 1 / 3, 0.0]),
    (False, True, [9.0, 6.5, 6.5, 9.0, 0.0], [12.5, 6.25, 11.25, 10.0, 0.0]),
    (False, False, [3.0, 0.5, 0.5, 3.0, 0.0], [4.0, 1.0, 2.0, 4.0, 0.0]),
]


def betweenness_example():
    # compute/centrality/tests.rs:79-85: 0 → 1 → 2 → 3 → 0, 0 → 2, 1 → 3, node 4 alone.
    return directed(5, [(0, 1), (1, 2), (2, 3), (0, 2), (3, 0), (1, 3)])


def test_betweenness_known_answers(oracle):
    g = betweenness_example()
    every = O.sample_sources(5)
    two = O.sample_sources(5, population=np.array([1, 0, 1, 0, 0]))
    for normalized, endpoints, exact, from_two in BETWEENNESS_KATS:
        got = O.betweenness(g, every, normalized=normalized, endpoints=endpoints)
        assert np.allclose(got, exact, rtol=1e-12, atol=0), (normalized, endpoints)
        got = O.betweenness(g, two, normalized=normalized, endpoints=endpoints)
        assert np.allclose(got, from_two, rtol=1e-12, atol=0), (normalized, endpoints)
