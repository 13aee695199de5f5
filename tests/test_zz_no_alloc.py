"""wc_pagerank_noalloc (no reference counterpart): PageRank whose working
memory is the library's fixed device array, for callers that cannot
allocate device memory while they serve a query.  Two calls in a row must
equal wc_pagerank on the same version (same kernels in the same order:
equal iteration counts and equal ranks, bit for bit); a call on a freshly
uploaded version must leave its budget's bytes in use and peak unchanged;
sizes past the array's 64 MiB are refused with WorkingSet before anything
runs.

The file is named to be collected last, so that it also runs after every
other GPU test has used the same process."""

import numpy as np
import pytest

import pg_warren_b200 as W

pytestmark = pytest.mark.gpu

LIMIT = 64 << 20


@pytest.mark.parametrize("weighted", [False, True])
def test_two_calls_in_a_row_equal_wc_pagerank(weighted):
    g = W.rmat(15, seed=5)
    if weighted:
        g.weights = W.edge_weights(g, "uniform")
    gv = g.upload()
    opts = W.PageRank(0.85, 1e-9, 100)
    ref = W.pagerank(gv, None, opts)
    for _ in range(2):
        r = W.pagerank_noalloc(gv, None, opts)
        assert r.iterations == ref.iterations
        assert np.array_equal(r.values, ref.values)
    assert W.last_margin(gv) > 0.0


def test_a_call_charges_no_memory_to_the_budget():
    # The property the entry point exists for: on a freshly uploaded version
    # (no pooled scratch yet) the call takes no device memory, so the budget
    # the version is charged to is left as it was; wc_pagerank on the same
    # version then charges its own scratch and gives the same ranks.
    budget = W.Budget()
    g = W.rmat(14, seed=3)
    gv = W.GraphVersion(g.offsets, g.targets, budget=budget)
    in_use, peak = budget.in_use, budget.peak
    info = gv.info()
    held = (info.device_bytes, info.scratch_bytes)
    opts = W.PageRank(0.85, 1e-10, 100)
    for _ in range(2):
        r = W.pagerank_noalloc(gv, None, opts)
        assert (budget.in_use, budget.peak) == (in_use, peak)
        info = gv.info()
        assert (info.device_bytes, info.scratch_bytes) == held
    ref = W.pagerank(gv, None, opts)
    assert budget.in_use > in_use and gv.info().scratch_bytes > held[1]
    assert r.iterations == ref.iterations and np.array_equal(r.values, ref.values)


def test_the_progress_hook_runs_outside_the_locks():
    # A hook that itself calls the entry point on the same device must not
    # wait on the call that invoked it.
    g = W.rmat(10, seed=4)
    gv, inner = g.upload(), g.upload()
    opts = W.PageRank(0.85, 1e-10, 100)
    seen = []

    def hook(phase, done, total):
        if not seen:
            seen.append(W.pagerank_noalloc(inner, None, opts).iterations)
        seen.append(done)

    r = W.pagerank_noalloc(gv, None, opts, interrupts=W.Interrupts(progress=hook))
    ref = W.pagerank(gv, None, opts)
    assert seen == [ref.iterations, 0, ref.iterations]
    assert np.array_equal(r.values, ref.values)


def test_tombstones_on_host_and_device():
    torch = pytest.importorskip("torch")
    g = W.rmat(12, seed=9)
    gv = g.upload()
    tomb = W.node_set(g.id_space, range(0, g.id_space, 7))
    opts = W.PageRank(0.85, 1e-10, 200)
    ref = W.pagerank(gv, tomb, opts)
    a = W.pagerank_noalloc(gv, tomb, opts)
    td = torch.from_numpy(tomb.view(np.int64)).cuda()
    b = W.pagerank_noalloc(gv, td, opts)
    for r in (a, b):
        assert r.iterations == ref.iterations
        assert np.array_equal(r.values, ref.values)
        assert np.all(r.values[::7] == 0.0)


def test_fixed_iteration_count_and_no_iterations():
    g = W.rmat(10, seed=2)
    gv = g.upload()
    for opts in (W.PageRank(tol=None, max_iter=7), W.PageRank(max_iter=0)):
        ref = W.pagerank(gv, None, opts)
        r = W.pagerank_noalloc(gv, None, opts)
        assert r.iterations == ref.iterations
        assert np.array_equal(r.values, ref.values)


def test_sizes_past_the_array_are_refused():
    n = 1_700_000  # 40 bytes a node: 68 MB > 64 MiB
    gv = W.GraphVersion(np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32))
    with pytest.raises(W.api.WorkingSet) as e:
        W.pagerank_noalloc(gv, None, W.PageRank())
    assert e.value.detail.limit == LIMIT and e.value.detail.requested > LIMIT
    # The existing entry point still serves it.
    r = W.pagerank(gv, None, W.PageRank(max_iter=3))
    assert r.iterations >= 1


def test_personalised_solves_are_not_offered():
    g = W.rmat(8, seed=1)
    gv = g.upload()
    seed = np.ones(g.id_space)
    with pytest.raises(W.api.Unsupported):
        W.pagerank_noalloc(gv, None, W.PageRank(seed=seed))
