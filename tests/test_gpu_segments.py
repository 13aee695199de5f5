"""A version loaded from its stored segments (wc_version_load_segments)
against one uploaded from arrays, the reverse CSR built on the device, and
the CSR checks that run on the device, each reporting the first violation
in the reference's order (graph/csr/mod.rs:78-137)."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W
from pg_warren_b200 import api

pytestmark = pytest.mark.gpu


def load(n, off, tgt, w=None, rows=None, reverse=True):
    o = api.encode_segment(1, np.asarray(off, np.uint64))
    t = api.encode_segment(2, np.asarray(tgt, np.uint32))
    ws = None if w is None else api.encode_segment(3, np.asarray(w, np.float64))
    rs = None if rows is None else api.encode_segment(11, np.asarray(rows, np.uint32))
    return W.GraphVersion.from_segments(n, o, t, ws, rs, reverse=reverse)


@pytest.mark.parametrize("sparse", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
def test_segments_give_the_arrays_version(sparse, weighted):
    g = W.rmat(12, seed=3)
    w = W.edge_weights(g, "int") if weighted else None
    rows, off, tgt, ws = api.csr_segments(g.offsets, g.targets, w, sparse=sparse)
    if sparse:
        assert rows is not None and len(rows) < 16 + 4 * g.id_space
    gs = W.GraphVersion.from_segments(g.id_space, off, tgt, ws, rows)
    ga = W.GraphVersion(g.offsets, g.targets, w)
    gh = W.GraphVersion(g.offsets, g.targets, w, reverse=W.api.host_reverse(g.offsets, g.targets, w))
    ia, ib, ih = ga.info(), gs.info(), gh.info()
    facts = lambda i: (i.id_space, i.edges, i.weighted, i.integral_weights, i.symmetric)
    assert facts(ia) == facts(ib) == facts(ih)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w)
    rng = np.random.default_rng(1)
    x = rng.integers(0, 5, g.id_space).astype(np.float64)
    for transpose in (False, True):
        yo = np.zeros(g.id_space)
        O.product(og, 0, x, yo, transpose=transpose)
        for gv in (gs, ga, gh):
            y = np.zeros(g.id_space)
            W.spmv(gv, W.Product("plus_times", transpose=transpose), x, y)
            assert y.tobytes() == yo.tobytes(), transpose
    d1 = W.bfs_depths(gs, [0, 5], direction="in")
    d2 = W.bfs_depths(gh, [0, 5], direction="in")
    assert np.array_equal(d1[0], d2[0]) and np.array_equal(d1[1], d2[1])


def test_without_a_reverse_in_searches_are_refused():
    gv = load(3, [0, 2, 2, 4], [1, 2, 0, 2], reverse=False)
    with pytest.raises(api.ReverseCsrMissing):
        W.bfs_depths(gv, [0], direction="in")
    W.bfs_depths(gv, [0], direction="out")


def detail(exc):
    d = exc.value.detail
    return d.node, d.expected, d.found


def test_device_checked_errors_in_the_references_order():
    with pytest.raises(api.StoredRowsNotAscending) as e:
        load(5, [0, 1, 2, 3], [1, 2, 3], rows=[0, 3, 3])
    assert detail(e)[0] == 2
    with pytest.raises(api.StoredRowOutsideIdSpace) as e:
        load(5, [0, 1, 2], [1, 2], rows=[0, 7])
    assert detail(e)[0] == 7
    with pytest.raises(api.StoredRowEmpty) as e:
        load(5, [0, 1, 1, 2], [1, 2], rows=[0, 2, 3])
    assert detail(e)[0] == 2
    with pytest.raises(api.OffsetsNotMonotone) as e:
        load(3, [0, 2, 1, 3], [1, 2, 0])
    assert detail(e)[0] == 1
    with pytest.raises(api.FinalOffset) as e:
        load(3, [0, 1, 2, 2], [1, 2, 0])
    assert detail(e)[1:] == (3, 2)
    with pytest.raises(api.TargetOutsideIdSpace) as e:
        load(3, [0, 1, 3, 4], [1, 0, 9, 1])
    assert detail(e)[0] == 1 and detail(e)[2] == 9
    with pytest.raises(api.RowNotSorted) as e:
        load(3, [0, 2, 3, 4], [2, 1, 0, 1])
    assert detail(e)[0] == 0
    # Row 0 unsorted comes before row 2's outside target; in one row, the
    # outside target comes first.
    with pytest.raises(api.RowNotSorted) as e:
        load(3, [0, 2, 2, 3], [2, 1, 7])
    assert detail(e)[0] == 0
    with pytest.raises(api.TargetOutsideIdSpace) as e:
        load(3, [0, 3, 3, 3], [2, 1, 7])
    assert detail(e)[0] == 0
    with pytest.raises(api.WeightsLength) as e:
        load(3, [0, 1, 2, 2], [1, 2], w=[1.0])
    assert detail(e)[1:] == (2, 1)


def test_empty_and_edge_free_versions():
    gv = load(4, [0, 0, 0, 0, 0], [])
    assert gv.info().edges == 0
    gv = load(4, [0], [], rows=[])
    assert gv.info().edges == 0 and gv.info().id_space == 4
    y = np.zeros(4)
    W.spmv(gv, W.Product("plus_times", transpose=True), np.ones(4), y)
    assert not y.any()


def test_device_transpose_keeps_duplicate_entries_in_order():
    # Duplicate (source, target) entries whose sum depends on their order:
    # the reverse rows keep them in forward order, as the counting
    # transpose does.
    off = np.array([0, 3, 5, 6], np.uint64)
    tgt = np.array([1, 1, 2, 0, 2, 1], np.uint32)
    w = np.array([1e16, 1.0, -3.0, 2.0, 0.5, -1e16])
    og = O.Graph.from_csr(3, off, tgt, w)
    gv = W.GraphVersion(off, tgt, w)
    x = np.array([1.0, 1.0, 1.0])
    y = np.zeros(3)
    W.spmv(gv, W.Product("plus_times", transpose=True), x, y)
    yo = np.zeros(3)
    O.product(og, 0, x, yo, transpose=True)
    assert y.tobytes() == yo.tobytes()
