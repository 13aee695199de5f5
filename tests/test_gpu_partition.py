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
