"""The runtime contract on the device (compute/memory.rs, interrupts.rs):
budget refusals carry what was asked, what is held and the limit; a cancel
raised from another thread while a call runs ends it with Cancelled; a wait
past the call's timeout ends it with DeviceTimeout, and a device-side wait
that runs out ends with a status, the device staying usable; the device's
seeded start vectors equal the reference's generator bit for bit."""

import threading
import time

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu


def unweighted(scale, seed=1, budget=None, reverse=True):
    g = W.rmat(scale, seed=seed)
    if reverse is not True:
        reverse = W.api.host_reverse(g.offsets, g.targets)
    return g, W.GraphVersion(g.offsets, g.targets, reverse=reverse, budget=budget)


def test_a_call_budget_below_its_working_memory_is_memory_limit():
    # memory.rs:140-171 (try_reserve), test :472: MemoryLimit {requested,
    # in_use, limit}; nothing is charged for the refused call.
    g, gv = unweighted(12)
    n = g.id_space
    budget = W.Budget(1000)
    with pytest.raises(W.MemoryLimit) as e:
        W.pagerank(gv, None, W.PageRank(), memory=budget)
    d = e.value.detail
    assert (d.in_use, d.limit) == (0, 1000)
    assert d.requested == 2 * n * 8  # the two rank vectors, the first buffer asked for
    assert budget.in_use == 0
    # A budget with room serves the call and holds nothing after it.
    roomy = W.Budget(1 << 30)
    r = W.pagerank(gv, None, W.PageRank(), memory=roomy)
    assert r.iterations > 0 and roomy.in_use == 0 and roomy.peak >= 5 * n * 8
    # The batched search is refused the same way.
    with pytest.raises(W.MemoryLimit):
        W.bfs_batched(gv, [0, 1], [3, 3], memory=W.Budget(4096))


def test_a_version_budget_with_no_room_left_is_memory_limit():
    # The device copy fills its budget exactly (the reverse given, so the
    # upload needs no transient room); the first call's scratch is refused.
    probe = W.Budget()
    unweighted(12, budget=probe, reverse=False)
    budget = W.Budget(probe.peak)
    g, gv = unweighted(12, budget=budget, reverse=False)
    held = budget.in_use
    assert held <= probe.peak and probe.peak - held < 2 * g.id_space * 8
    with pytest.raises(W.MemoryLimit) as e:
        W.pagerank(gv, None, W.PageRank())
    d = e.value.detail
    assert d.in_use == held and d.limit == probe.peak and d.requested >= 2 * g.id_space * 8
    assert budget.in_use == held


def test_a_version_keeps_its_budget_after_the_caller_drops_it():
    # The caller may destroy a budget before the versions charged to it are
    # released (a garbage collector finalises them in any order): the
    # version holds the budget until its own buffers are freed.
    budget = W.Budget()
    g, gv = unweighted(12, budget=budget)
    held = budget.in_use
    handle, budget.handle = budget.handle, None
    W.load().wc_budget_destroy(handle)  # the caller's hold goes first
    r = W.pagerank(gv, None, W.PageRank())  # scratch charged to the budget
    assert r.iterations > 0 and held > 0
    gv.release()  # frees the buffers, uncharges, then lets the budget go
    g2, gv2 = unweighted(12)
    assert W.pagerank(gv2, None, W.PageRank()).iterations == r.iterations


def test_cancel_from_another_thread_during_pagerank():
    # interrupts.rs:52-120: a flag raised on one thread while the work polls
    # it on another.  5,000 iterations without a tolerance: far longer than
    # the 20 ms after which the flag is raised.
    g, gv = unweighted(18)
    intr = W.Interrupts(progress=lambda phase, done, total: started.set())
    started = threading.Event()

    def raise_flag():
        started.wait(30)
        time.sleep(0.02)
        intr.cancel()

    t = threading.Thread(target=raise_flag)
    t.start()
    t0 = time.perf_counter()
    with pytest.raises(W.Cancelled):
        W.pagerank(gv, None, W.PageRank(0.85, None, 5000), interrupts=intr)
    t.join()
    # The kernels stopped at the flag rather than running every iteration.
    full = time.perf_counter()
    r = W.pagerank(gv, None, W.PageRank(0.85, None, 5000))
    assert r.iterations == 5000
    assert full - t0 < 0.9 * (time.perf_counter() - full) + 0.05
    # The version serves the next call normally.
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets)
    ro, it, _, _ = O.pagerank(og, 0.85, 1e-10, 100)
    r = W.pagerank(gv, None, W.PageRank(0.85, 1e-10, 100))
    assert r.iterations == it and np.abs(r.values - ro).sum() / ro.sum() <= 1e-12


def test_cancel_from_another_thread_during_a_batched_search():
    torch = pytest.importorskip("torch")
    g, gv = unweighted(18)
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, reverse=False)
    rng = np.random.default_rng(5)
    src = rng.integers(0, g.id_space, 8192).astype(np.uint64)
    caps = np.full(8192, 16, np.uint32)
    intr = W.Interrupts()
    go = threading.Event()

    def raise_flag():
        go.wait(30)
        time.sleep(0.03)
        intr.cancel()

    t = threading.Thread(target=raise_flag)
    t.start()
    go.set()
    with pytest.raises(W.Cancelled):
        W.bfs_batched(gv, src, caps, interrupts=intr)  # 8 passes, depths copied to the host
    t.join()
    # The accumulators the search keeps zero between calls are still zero:
    # the next call is exact.
    d, e = W.bfs_batched(gv, src[:300], caps[:300])
    do, eo = O.bfs_depths(og, src[:300], caps[:300])
    assert np.array_equal(d, do) and np.array_equal(e, eo)
    del torch


def test_a_call_past_its_timeout_is_device_timeout():
    g, gv = unweighted(18)
    with pytest.raises(W.DeviceTimeout):
        W.pagerank(gv, None, W.PageRank(0.85, None, 2000), timeout_ms=1)
    r = W.pagerank(gv, None, W.PageRank(0.85, None, 5))
    assert r.iterations == 5


def test_a_device_wait_that_runs_out_returns_a_status():
    # The bounded wait of the bulk-copy rings on a barrier nothing completes:
    # it gives up after the limit, the kernel returns, the call reports it.
    t0 = time.perf_counter()
    with pytest.raises(W.DeviceTimeout):
        W.selftest_bounded_wait(50_000)
    assert time.perf_counter() - t0 >= 0.05
    g, gv = unweighted(10)
    r = W.pagerank(gv, None, W.PageRank(max_iter=3, tol=None))
    assert r.iterations == 3


@pytest.mark.parametrize("seed,stream", [(1, 0), (7, 0), (7, 3), (2**64 - 1, 2**63)])
def test_device_start_vectors_equal_the_reference_generator(seed, stream):
    # compute/random.rs:11-25, the values pinned against random.rs:31-46 in
    # the oracle's own known-answer tests.
    n = 70_001
    gv = W.GraphVersion(np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32))
    got = W.random_uniform(gv, seed, stream)
    want = np.array([O.uniform(seed, stream, i) for i in range(n)])
    assert got.tobytes() == want.tobytes()
