"""The row-partitioned PageRank's device parts (wc_pagerank_part_*): one
part equals wc_pagerank; two parts of a solve, run on one GPU with the
exchange between them done by hand (what the ranks' collectives do), equal
it within the PageRank tolerance with equal iteration counts."""

import numpy as np
import pytest

import pg_warren_b200 as W
from pg_warren_b200.partition import DeviceParts, pagerank_partitioned

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


@pytest.mark.parametrize("scale,tol", [(12, 1e-10), (16, 1e-10), (14, None)])
def test_one_part_equals_pagerank(scale, tol):
    g = W.rmat(scale, seed=3)
    gv = g.upload()
    pr = W.PageRank(0.85, tol, 100 if tol else 9)
    want = W.pagerank(gv, None, pr)
    got = pagerank_partitioned(gv, None, pr)
    assert got.iterations == want.iterations
    assert rel_l1(got.values, want.values) <= 1e-14


@pytest.mark.parametrize("weighted", [False, True])
def test_two_parts_exchanging_by_hand_equal_pagerank(weighted):
    import torch
    g = W.rmat(15, seed=8)
    if weighted:
        g.weights = W.edge_weights(g, "uniform")
    tomb = W.node_set(g.id_space, range(0, g.id_space, 11))
    pr = W.PageRank(0.85, 1e-10, 100)
    want = W.pagerank(g.upload(), tomb, pr)
    versions = [g.upload(), g.upload()]
    parts = [DeviceParts(v, tomb, pr) for v in versions]
    bounds = parts[0].rows(2)
    assert bounds[0] == 0 and bounds[-1] == g.id_space and bounds[0] < bounds[1] < bounds[2]
    infos = [p.begin(2, k) for k, p in enumerate(parts)]
    assert [(i.row_begin, i.row_end) for i in infos] == [(bounds[0], bounds[1]), (bounds[1], bounds[2])]
    dangling, its = infos[0].dangling, 0
    assert infos[1].dangling == dangling
    for it in range(pr.max_iter):
        sums = [p.step(it, dangling) for p in parts]
        delta = sums[0][0] + sums[1][0]
        dangling = sums[0][1] + sums[1][1]
        nxt = (it + 1) & 1
        for k in range(2):  # part k's rows to the other part
            b, e = int(bounds[k]), int(bounds[k + 1])
            parts[1 - k].messages2[nxt][b:e] = parts[k].messages2[nxt][b:e]
        its = it + 1
        if delta < infos[0].threshold:
            break
    for k in range(2):
        b, e = int(bounds[k]), int(bounds[k + 1])
        parts[1 - k].ranks2[its & 1][b:e] = parts[k].ranks2[its & 1][b:e]
    torch.cuda.synchronize()
    got = [p.end(its) for p in parts]
    assert its == want.iterations
    for r in got:
        assert rel_l1(r, want.values) <= 1e-12
        assert np.all(r[::11] == 0.0)


# ----------------------------------------------- row-partitioned level search

UNREACHED = 0xFFFFFFFF


def oracle_depths(g, starts, direction, max_depth):
    import oracle as O
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    visits, _ = O.bfs(og, starts, {"out": 0, "in": 1, "both": 2}[direction], max_depth)
    want = np.full(g.id_space, UNREACHED, np.uint32)
    for node, depth, _ in visits:
        want[node] = depth
    return want


@pytest.mark.parametrize("direction,max_depth", [("out", None), ("in", 2), ("both", None),
                                                 ("out", 0)])
def test_one_search_part_equals_the_level_search(direction, max_depth):
    from pg_warren_b200.partition import bfs_partitioned
    g = W.rmat(14, seed=6)
    gv = g.upload()
    starts = [3, 77, 3, g.id_space - 1]
    depth, levels = bfs_partitioned(gv, starts, max_depth, direction)
    want = oracle_depths(g, starts, direction, max_depth)
    assert np.array_equal(depth, want)
    d, _, _ = W.bfs_depths(gv, starts, max_depth, direction)
    assert np.array_equal(depth, d)


@pytest.mark.parametrize("direction", ["out", "both"])
def test_two_search_parts_exchanging_by_hand_equal_the_level_search(direction):
    import torch
    from pg_warren_b200.partition import BfsDeviceParts
    g = W.rmat(15, seed=12)
    starts = [int(s) for s in np.random.default_rng(4).integers(0, g.id_space, 5)]
    parts = [BfsDeviceParts(g.upload(), starts, None, direction) for _ in range(2)]
    bounds = parts[0].rows(2)
    assert bounds[0] == 0 and bounds[-1] == g.id_space and bounds[1] % 64 == 0
    wb = [(int(b) + 63) // 64 for b in bounds]
    infos = [p.begin(2, k) for k, p in enumerate(parts)]
    assert [(i.row_begin, i.row_end) for i in infos] == [(bounds[0], bounds[1]),
                                                         (bounds[1], bounds[2])]
    count, edges = infos[0].frontier, infos[0].frontier_edges
    assert (infos[1].frontier, infos[1].frontier_edges) == (count, edges)
    level = 0
    while count:
        sums = [p.step(level, edges) for p in parts]
        count, edges = sums[0][0] + sums[1][0], sums[0][1] + sums[1][1]
        for k in range(2):  # part k's words of the next frontier to the other part
            parts[1 - k].frontier(level + 1)[wb[k]:wb[k + 1]] = \
                parts[k].frontier(level + 1)[wb[k]:wb[k + 1]]
        level += 1
    depths = [p.end() for p in parts]
    torch.cuda.synchronize()
    got = np.concatenate([depths[0][: bounds[1]].cpu().numpy(),
                          depths[1][bounds[1]:].cpu().numpy()]).view(np.uint32)
    want = oracle_depths(g, starts, direction, None)
    assert np.array_equal(got, want)
    assert level == int(want[want != UNREACHED].max()) + 1


def test_search_starts_outside_the_id_space_are_refused():
    from pg_warren_b200.partition import BfsDeviceParts
    g = W.rmat(8, seed=1)
    parts = BfsDeviceParts(g.upload(), [g.id_space], None, "out")
    with pytest.raises(W.api.NodeOutsideIdSpace):
        parts.begin(1, 0)


# -------------------------------------------------- row-partitioned products


@pytest.mark.parametrize("semiring,dtype,transpose,parts_n",
                         [("plus_times", np.float64, False, 2), ("plus_times", np.float64, True, 3),
                          ("min_plus", np.int64, True, 2), ("lor_land", np.bool_, False, 4)])
def test_product_parts_equal_spmv_bit_for_bit(semiring, dtype, transpose, parts_n):
    import torch
    from pg_warren_b200.partition import SpmvDeviceParts
    g = W.rmat(14, seed=9)
    if semiring != "lor_land":
        g.weights = W.edge_weights(g, "int" if dtype == np.int64 else "uniform")
    gv = g.upload()
    rng = np.random.default_rng(2)
    n = g.id_space
    if dtype == np.bool_:
        x = rng.random(n) < 0.1
    elif dtype == np.int64:
        x = rng.integers(0, 1000, n).astype(np.int64)
    else:
        x = rng.random(n)
    prod = W.Product(semiring, transpose=transpose)
    want = np.zeros(n, dtype)
    W.spmv(gv, prod, x, want)
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(np.zeros(n, dtype)).cuda()
    parts = SpmvDeviceParts(gv, prod)
    bounds = parts.rows(parts_n)
    assert bounds[0] == 0 and bounds[-1] == n and np.all(np.diff(bounds) >= 0)
    for k in range(parts_n):
        before = yd.clone()
        parts.apply(parts_n, k, xd, yd)
        changed = (yd != before).nonzero().flatten().cpu().numpy()
        assert np.all((changed >= bounds[k]) & (changed < bounds[k + 1]))
    assert np.array_equal(yd.cpu().numpy(), want)


def test_product_parts_keep_the_mask_and_accumulate():
    import torch
    from pg_warren_b200.partition import spmv_partitioned, SpmvDeviceParts
    g = W.rmat(13, seed=5)
    g.weights = W.edge_weights(g, "uniform")
    gv = g.upload()
    rng = np.random.default_rng(8)
    n = g.id_space
    x, y0 = rng.random(n), rng.random(n)
    mask = (rng.random(n) < 0.5).astype(np.float64)
    prod = W.Product("plus_times", transpose=True, mask=torch.from_numpy(mask).cuda(),
                     accumulate="plus")
    want = y0.copy()
    W.spmv(gv, W.Product("plus_times", transpose=True, mask=mask, accumulate="plus"), x, want)
    yd = torch.from_numpy(y0.copy()).cuda()
    parts = SpmvDeviceParts(gv, prod)
    for k in range(3):
        parts.apply(3, k, torch.from_numpy(x).cuda(), yd)
    assert np.array_equal(yd.cpu().numpy(), want)
    # One part (no process group) through the driver.
    yd = torch.from_numpy(y0.copy()).cuda()
    res = spmv_partitioned(gv, prod, torch.from_numpy(x).cuda(), yd)
    assert np.array_equal(res.cpu().numpy(), want)


def test_more_product_parts_than_units_leave_the_empty_parts_idle():
    import torch
    from pg_warren_b200.partition import SpmvDeviceParts
    g = W.rmat(4, seed=2)
    gv = g.upload()
    n = g.id_space
    x = np.arange(n, dtype=np.float64)
    want = np.zeros(n)
    W.spmv(gv, W.Product("plus_times"), x, want)
    parts = SpmvDeviceParts(gv, W.Product("plus_times"))
    yd = torch.zeros(n, dtype=torch.float64, device="cuda")
    for k in range(16):
        parts.apply(16, k, torch.from_numpy(x).cuda(), yd)
    assert np.array_equal(yd.cpu().numpy(), want)
