"""The C-ABI library on CPU: it loads without a GPU and exports every entry
point include/warren_cuda.h declares; graph synthesis (host code) matches
the oracle's build of the same edges."""

import ctypes
import os
import re

import numpy as np

import oracle as O
import pg_warren_b200 as W
from pg_warren_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "warren_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(_abi.LIBRARY)
    names = declared()
    assert len(names) >= 29
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_every_declared_entry_point_has_a_python_signature():
    bound = {name for name, _, _ in _abi.SIGNATURES}
    assert [n for n in declared() if n not in bound] == []


def test_status_names_and_serves():
    lib = _abi.load()
    assert lib.wc_status_name(13) == b"division by zero"
    assert lib.wc_status_name(10) == b"bigint out of range"
    assert lib.wc_serves(b"spmv", _abi.F64) == 1
    assert lib.wc_serves(b"pagerank", _abi.BOOL) == 0


def test_rmat_is_deterministic_deduplicated_and_sorted():
    g1 = W.rmat(12, seed=1)
    g2 = W.rmat(12, seed=1)
    assert np.array_equal(g1.offsets, g2.offsets) and np.array_equal(g1.targets, g2.targets)
    assert g1.id_space == 4096
    for r in range(g1.id_space):
        row = g1.targets[g1.offsets[r]:g1.offsets[r + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)  # ascending, distinct
        assert r not in row  # no self-loops
    # External ids are distinct and their sorted order is the dense order.
    assert np.all(np.diff(g1.external_ids) > 0)
    assert not np.array_equal(W.rmat(12, seed=2).targets[:100], g1.targets[:100])


def test_host_transpose_matches_the_oracle_reverse_csr(oracle):
    g = W.rmat(11, seed=3)
    w = W.edge_weights(g, "uniform")
    og = O.Graph.from_csr(g.id_space, g.offsets, g.targets, w, reverse=True)
    _, _, _, roff, rtgt, rw = og.csr()
    n, m = g.id_space, g.edges
    r_off = np.zeros(n + 1, np.uint64)
    r_tgt = np.zeros(m, np.uint32)
    r_w = np.zeros(m, np.float64)
    assert _abi.load().wc_host_transpose(n, m, g.offsets.ctypes.data, g.targets.ctypes.data,
                                         w.ctypes.data, r_off.ctypes.data, r_tgt.ctypes.data,
                                         r_w.ctypes.data) == 0
    assert np.array_equal(r_off, roff) and np.array_equal(r_tgt, rtgt)
    assert r_w.tobytes() == rw.tobytes()


def test_synthesis_equals_the_oracle_build_of_the_same_edges(oracle):
    # The oracle restates the reference's build (sort, fold repeats); fed the
    # product graph's own edges in a shuffled order with repeats, it must give
    # the same CSR back.
    g = W.gnm(3000, 20000, seed=5)
    src = np.repeat(np.arange(g.id_space), np.diff(g.offsets).astype(np.int64))
    edges = [(0, int(s), int(t), 1.0) for s, t in zip(src, g.targets)]
    rng = np.random.default_rng(0)
    extra = [edges[i] for i in rng.integers(0, len(edges), 500)]
    alle = edges + extra
    rng.shuffle(alle)
    og = O.Graph.from_edges(g.id_space, alle, weighted=False, reverse=False)
    off, tgt, _, _, _, _ = og.csr()
    assert np.array_equal(off, g.offsets) and np.array_equal(tgt, g.targets)
