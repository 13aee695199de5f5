"""vector_reduce / vector_norm_diff on the device against the oracle's
restatement of compute/reduce.rs: bit for bit, including the order of the
chunked float sums, NaN, signed zeros and tombstoned rows."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu

REDUCTIONS = ("sum", "max", "min", "l1", "l2", "nnz")


def same(a, b):
    if a is None or b is None:
        return a is None and b is None
    return np.float64(a).tobytes() == np.float64(b).tobytes()


def version(n):
    off = np.zeros(n + 1, np.uint64)
    return W.GraphVersion(off, np.zeros(0, np.uint32))


def values(rng, dtype, size):
    if dtype == np.float64:
        x = rng.standard_normal(size) * 10.0 ** rng.integers(-12, 13, size)
        x[rng.random(size) < 0.01] = np.nan
        x[rng.random(size) < 0.01] = -0.0
        x[rng.random(size) < 0.01] = 0.0
        return x
    if dtype == np.float32:
        return rng.standard_normal(size).astype(np.float32)
    if dtype == np.int64:
        return rng.integers(-2**62, 2**62, size)
    return rng.random(size) < 0.3


@pytest.mark.parametrize("n,width", [(0, 1), (1, 1), (5, 3), (70_000, 1), (300_001, 1),
                                     (100_000, 3)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int64, np.bool_])
def test_reductions_match_the_oracle(n, width, dtype):
    rng = np.random.default_rng(n + width)
    gv = version(n)
    x = values(rng, dtype, n * width)
    x2 = x.reshape(n, width) if width > 1 else x
    tomb = W.node_set(n, rng.integers(0, max(n, 1), n // 10)) if n else None
    for r in REDUCTIONS:
        assert same(W.vector_reduce(gv, x2, r), O.reduce(x, r, width)), (r, dtype)
        assert same(W.vector_reduce(gv, x2, r, tombstones=tomb),
                    O.reduce(x, r, width, tombstones=tomb)), (r, dtype, "live")


def test_the_reference_examples():
    gv = version(2)
    found = [W.vector_reduce(gv, np.array([[3.0, -4.0], [0.0, 1.0]]), r) for r in REDUCTIONS]
    assert found == [0.0, 3.0, -4.0, 8.0, 26 ** 0.5, 3.0]
    gv3 = version(3)
    x = np.array([1.0, np.nan, -2.0])
    assert np.isnan(W.vector_reduce(gv3, x, "max")) and W.vector_reduce(gv3, x, "min") == -2.0
    assert W.vector_reduce(version(0), np.zeros(0), "max") is None
    old, new = np.array([1.0, 2.0]), np.array([1.0, 5.0, -4.0])
    assert W.vector_norm_diff(gv3, new, old, "l1") == 7.0
    assert W.vector_norm_diff(gv3, old, new, "l2") == 5.0
    assert W.vector_norm_diff(gv3, old, new, "linf") == 4.0
    assert W.vector_norm_diff(gv3, np.array([1, 2], np.int64), old, "l1") == 0.0
    assert W.vector_norm_diff(gv3, np.zeros(0), np.zeros(0), "linf") == 0.0
    with pytest.raises(W.api.WidthMismatch):
        W.vector_norm_diff(gv3, np.ones((2, 2)), np.ones(2), "l1")


@pytest.mark.parametrize("na,nb", [(200_000, 150_001), (3, 70_000), (0, 10)])
def test_norm_diff_matches_the_oracle(na, nb):
    rng = np.random.default_rng(na + nb)
    gv = version(4)
    a, b = values(rng, np.float64, na), values(rng, np.float64, nb)
    for norm in ("l1", "l2", "linf"):
        assert same(W.vector_norm_diff(gv, a, b, norm), O.norm_diff(a, b, norm)), norm
    bi = rng.integers(-1000, 1000, nb)
    assert same(W.vector_norm_diff(gv, a, bi, "l2"), O.norm_diff(a, bi, "l2"))


def test_device_operands():
    import torch
    rng = np.random.default_rng(9)
    x = values(rng, np.float64, 500_000)
    gv = version(len(x))
    xd = torch.as_tensor(x, device="cuda")
    for r in REDUCTIONS:
        assert same(W.vector_reduce(gv, xd, r), O.reduce(x, r))
