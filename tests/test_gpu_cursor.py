"""The level-at-a-time BFS cursor (traversal/bfs_cursor.rs) against the
oracle: each level's visits in the reference's order, the concatenation
equal to bfs / reachable_set, the stats after every level, max_results,
a visitor that breaks, argument checks and cancellation."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu

DIRS = {"out": 0, "in": 1, "both": 2}


def directed(n, pairs, reverse=True):
    og = O.Graph.from_edges(n, [(0, s, t, 1.0) for s, t in pairs], weighted=False)
    off, tgt, _, _, _, _ = og.csr()
    return og, W.GraphVersion(off, tgt, None, reverse=reverse)


def example():
    # bfs_cursor.rs tests: 0 → 1 → 2 → 3, 0 → 4 → 3, 2 → 2, 5 isolated
    return directed(6, [(0, 1), (1, 2), (2, 3), (0, 4), (4, 3), (2, 2)])


def levels(cursor):
    out = []
    while True:
        visits, more = cursor.next_level()
        if visits:
            out.append([(v.node, v.depth, v.via) for v in visits])
        if not more:
            return out


def stats_tuple(s):
    return (s.nodes_visited, s.edges_traversed, s.truncated)


def test_a_cursor_hands_out_the_bfs_one_level_at_a_time():
    og, gv = example()
    with W.BfsCursor(gv, [0]) as c:
        lv = levels(c)
        assert [len(x) for x in lv] == [1, 2, 2]
        expected, st = O.bfs(og, [0])
        assert sum(lv, []) == expected
        assert stats_tuple(c.stats()) == (st["nodes_visited"], st["edges_traversed"], False)


def test_a_cursor_applies_the_filter_and_the_limits_as_bfs_does():
    og, gv = example()
    with W.BfsCursor(gv, [0, 0], filter=[1, 2, 3], limits=W.Limits(2, 2)) as c:
        found = sum(levels(c), [])
        expected, st = O.bfs(og, [0, 0], max_depth=2, max_results=2, filter_ids=[1, 2, 3])
        assert found == expected
        assert c.stats().truncated
        assert stats_tuple(c.stats()) == (st["nodes_visited"], st["edges_traversed"], True)


def test_a_visitor_that_breaks_finishes_the_cursor_without_truncating_it():
    _, gv = example()
    with W.BfsCursor(gv, [0]) as c:
        assert c.next_level(lambda v: True) is False
        assert c.next_level(lambda v: False) is False
        assert c.stats().nodes_visited == 1
        assert not c.stats().truncated


def test_a_cursor_checks_its_arguments_up_front():
    _, gv = example()
    with pytest.raises(W.api.NodeOutsideIdSpace):
        W.BfsCursor(gv, [6])
    _, fwd_only = directed(6, [(0, 1)], reverse=False)
    with pytest.raises(W.api.ReverseCsrMissing):
        W.BfsCursor(fwd_only, [0], direction="in")
    with pytest.raises(W.api.InvalidArgument):
        W.BfsCursor(gv, [0], filter=[1], reachable=True)


def test_a_raised_cancellation_stops_the_cursor():
    _, gv = example()
    with W.BfsCursor(gv, [0]) as c:
        intr = W.Interrupts()
        intr.cancel()
        with pytest.raises(W.api.Cancelled):
            c.next_level(interrupts=intr)
        # the cancelled cursor is finished
        assert c.next_level() == ([], False)


def test_a_version_is_not_released_under_an_open_cursor():
    _, gv = example()
    c = W.BfsCursor(gv, [0])
    with pytest.raises(W.api.InvalidArgument):
        gv.release()
    c.close()
    gv.release()


def check_cursor(og, gv, starts, direction, filt, depth, results):
    ov, ost = O.bfs(og, starts, direction=DIRS[direction], max_depth=depth, max_results=results,
                    filter_ids=filt)
    with W.BfsCursor(gv, starts, filter=filt, limits=W.Limits(depth, results),
                     direction=direction) as c:
        lv = levels(c)
        assert sum(lv, []) == ov
        # a level holds one depth, the depths ascend one by one from 0
        assert [x[0][1] for x in lv] == list(range(len(lv)))
        assert all(len({v[1] for v in x}) == 1 for x in lv)
        assert stats_tuple(c.stats()) == (ost["nodes_visited"], ost["edges_traversed"],
                                          ost["truncated"])


def check_reachable_cursor(og, gv, starts, direction, depth):
    nodes, ost = O.reachable_set(og, starts, direction=DIRS[direction], max_depth=depth)
    with W.BfsCursor.reachable_set(gv, starts, max_depth=depth, direction=direction) as c:
        visits = sum(levels(c), [])
        assert [v[0] for v in visits] == nodes
        st = c.stats()
        assert (st.nodes_visited, st.edges_traversed) == (ost["nodes_visited"],
                                                          ost["edges_traversed"])
        assert st.pulled_levels == ost["pulled_levels"]
    # depth is the BFS depth and via a node one level up with an edge to it
    ov, _ = O.bfs(og, starts, direction=DIRS[direction], max_depth=depth)
    depth_of = {a: b for a, b, _ in ov}
    off, tgt, _, roff, rtgt, _ = og.csr()
    for node, d, via in visits:
        assert depth_of[node] == d
        if via is not None:
            assert depth_of[via] == d - 1
            out_row = set(tgt[off[via]:off[via + 1]].tolist())
            in_row = set(rtgt[roff[via]:roff[via + 1]].tolist()) if roff is not None else set()
            row = {"out": out_row, "in": in_row, "both": out_row | in_row}[direction]
            assert node in row


def test_a_cursor_yields_exactly_the_bfs_random():
    rng = np.random.default_rng(11)
    for trial in range(20):
        n = int(rng.integers(3, 300))
        pairs = [(int(rng.integers(0, n)), int(rng.integers(0, n)))
                 for _ in range(int(rng.integers(0, 5 * n)))]
        og, gv = directed(n, pairs)
        starts = [int(v) for v in rng.integers(0, n, int(rng.integers(0, 3)))]
        for direction in ("out", "in", "both"):
            filt = [int(v) for v in rng.choice(n, n // 2, replace=False)] if trial % 3 == 0 else None
            depth = None if trial % 2 else int(rng.integers(0, 4))
            results = None if trial % 4 else int(rng.integers(0, 8))
            check_cursor(og, gv, starts, direction, filt, depth, results)
            check_reachable_cursor(og, gv, starts, direction, depth)


def test_a_visitor_that_breaks_anywhere_has_the_stats_of_the_search_up_to_there():
    # Breaking at the k-th visit admits it: nodes_visited k, and the entries
    # scanned are those through its entry, which a search limited to k - 1
    # results scans before it refuses that same visit.
    rng = np.random.default_rng(12)
    for trial in range(12):
        n = int(rng.integers(5, 200))
        pairs = [(int(rng.integers(0, n)), int(rng.integers(0, n))) for _ in range(4 * n)]
        og, gv = directed(n, pairs)
        starts = [int(rng.integers(0, n))]
        direction = ("out", "in", "both")[trial % 3]
        reachable = trial % 2 == 1
        full, _ = O.bfs(og, starts, direction=DIRS[direction], pulling=reachable)
        k = int(rng.integers(1, len(full) + 1))
        cut, cst = O.bfs(og, starts, direction=DIRS[direction], max_results=k - 1,
                         pulling=reachable)
        seen = []
        make = W.BfsCursor.reachable_set if reachable else W.BfsCursor
        with make(gv, starts, direction=direction) as c:
            def visitor(v):
                seen.append(v.node)
                return len(seen) == k
            while c.next_level(visitor):
                pass
            st = c.stats()
        assert seen == [v[0] for v in full[:k]]
        assert (st.nodes_visited, st.edges_traversed, st.truncated) == (k, cst["edges_traversed"],
                                                                        False)


def test_cursor_rmat16_with_pulled_levels():
    g = W.rmat(16, seed=1)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    for s in (0, 17, 4242):
        check_cursor(og, gv, [s], "out", None, 8, None)
        check_cursor(og, gv, [s], "out", None, None, 5000)
        nodes, ost = O.reachable_set(og, [s])
        with W.BfsCursor.reachable_set(gv, [s]) as c:
            assert [v[0] for v in sum(levels(c), [])] == nodes
            assert c.stats().pulled_levels == ost["pulled_levels"]
            assert c.stats().edges_traversed == ost["edges_traversed"]


def test_a_cursor_keeps_its_state_across_other_calls_on_the_version():
    # The cursor's buffers are its own: searches run on the same version
    # between its levels change nothing it hands out.
    g = W.rmat(14, seed=3)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    gv = W.GraphVersion(g.offsets, g.targets)
    expected, st = O.bfs(og, [5])
    with W.BfsCursor(gv, [5]) as c, W.BfsCursor.reachable_set(gv, [9]) as other:
        found = []
        more = True
        while more:
            visits, more = c.next_level()
            found += [(v.node, v.depth, v.via) for v in visits]
            W.bfs(gv, [int(len(found) % g.id_space)], limits=W.Limits(3, None))
            other.next_level()
        assert found == expected
        assert c.stats().edges_traversed == st["edges_traversed"]
