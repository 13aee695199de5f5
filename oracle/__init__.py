"""TEST INFRASTRUCTURE: the CPU oracle.

A ctypes binding of ``warren_oracle.cpp``, the C++ restatement of the
reference's warren-core kernels on the compute path (semirings, products,
PageRank, level-synchronous BFS and reachability, the ``sssp_vector`` loop,
Lanczos).  Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline use it, always as the checker or the baseline being timed; the
product (``pg_warren_b200``) never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCE = os.path.join(HERE, "warren_oracle.cpp")
# The benchmark graphs' generator (workload synthesis, not the compute path)
# is compiled into the oracle from the same source as into the CUDA library,
# so the CPU baseline builds its graph without mapping that library.
GRAPHGEN = os.path.join(HERE, "..", "pg_warren_b200", "csrc", "graphgen.cpp")
LIBRARY = os.path.join(HERE, "liboracle.so")

# Status codes shared with include/warren_cuda.h.
OK = 0

_lib = None


def build(force: bool = False) -> str:
    """Compiles the oracle (g++, -O3, threads) into oracle/liboracle.so."""
    deps = [SOURCE, os.path.join(HERE, "warren_lanczos.cpp"), GRAPHGEN,
            os.path.join(HERE, "..", "include", "warren_cuda.h")]
    deps = [d for d in deps if os.path.exists(d)]
    if not force and os.path.exists(LIBRARY):
        built = os.path.getmtime(LIBRARY)
        if all(os.path.getmtime(d) <= built for d in deps):
            return LIBRARY
    sources = [d for d in deps if d.endswith(".cpp")]
    cmd = ["g++", "-O3", "-std=c++17", "-shared", "-fPIC", "-Wall", "-Wno-maybe-uninitialized", "-o", LIBRARY + ".tmp",
           *sources, "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(LIBRARY + ".tmp", LIBRARY)
    return LIBRARY


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            build()
        _lib = C.CDLL(LIBRARY)
        _declare(_lib)
    return _lib


P = C.c_void_p
U64 = C.c_uint64
U32 = C.c_uint32
I32 = C.c_int32
I = C.c_int
D = C.c_double


def _declare(L):
    L.wo_graph_build.restype = P
    L.wo_graph_build.argtypes = [U64, U32, U64, P, P, P, P, I]
    L.wo_graph_from_csr.restype = P
    L.wo_graph_from_csr.argtypes = [U64, U64, P, P, P, I]
    L.wo_graph_free.argtypes = [P]
    L.wo_graph_edges.restype = U64
    L.wo_graph_edges.argtypes = [P]
    L.wo_graph_weighted.restype = I
    L.wo_graph_weighted.argtypes = [P]
    L.wo_graph_copy.argtypes = [P, P, P, P, P, P, P]
    L.wo_set_threads.argtypes = [I]
    L.wo_threads.restype = I
    L.wo_set_chunk.argtypes = [U64]
    L.wo_apply.restype = I32
    L.wo_apply.argtypes = [I, I, P, P, P]
    L.wo_multiply.restype = I32
    L.wo_multiply.argtypes = [I, I, I, P, P, P]
    L.wo_from_weight.restype = I32
    L.wo_from_weight.argtypes = [I, D, P]
    L.wo_identity.argtypes = [I, I, P]
    L.wo_semiring_add.restype = I
    L.wo_semiring_add.argtypes = [I]
    L.wo_semiring_mul.restype = I
    L.wo_semiring_mul.argtypes = [I]
    L.wo_float.restype = I32
    L.wo_float.argtypes = [I, D, D, C.POINTER(D)]
    L.wo_uniform.restype = D
    L.wo_uniform.argtypes = [U64, U64, U64]
    L.wo_product.restype = I32
    L.wo_product.argtypes = [P, I, I, I, P, I, I, I, I, I, U64, P, P, I]
    L.wo_pagerank.restype = I32
    L.wo_pagerank.argtypes = [P, P, D, I, D, I, U32, P, P, P, P, P]
    L.wo_bfs.restype = I32
    L.wo_bfs.argtypes = [P, I, P, U64, U32, U64, P, P, U64, P, P]
    L.wo_level_search.restype = I32
    L.wo_level_search.argtypes = [P, I, P, U64, U32, U64, P, I, P, U64, P, P]
    L.wo_reachable_set.restype = I32
    L.wo_reachable_set.argtypes = [P, I, P, U64, U32, P, U64, P, P]
    L.wo_bfs_depths.restype = I32
    L.wo_bfs_depths.argtypes = [P, P, P, U32, P, P]
    L.wo_bfs_depths_batched64.restype = I32
    L.wo_bfs_depths_batched64.argtypes = [P, P, P, U32, P, P]
    L.wo_sssp_i64.restype = I32
    L.wo_sssp_i64.argtypes = [P, P, P, U32, P, P]
    L.wo_components.restype = I32
    L.wo_components.argtypes = [P, P, P, P]
    L.wo_topk_f64.restype = I32
    L.wo_topk_f64.argtypes = [P, U64, P, U64, I, P, P, P]
    L.wo_reduce.restype = I32
    L.wo_reduce.argtypes = [I, P, U64, U64, P, I, P, P]
    L.wo_norm_diff.restype = I32
    L.wo_norm_diff.argtypes = [I, P, U64, I, P, U64, U64, I, P]
    L.wo_betweenness.restype = I32
    L.wo_betweenness.argtypes = [P, P, U64, P, I, I, I, P]
    L.wo_sample_sources.restype = I32
    L.wo_sample_sources.argtypes = [U64, P, P, I, C.c_int64, U64, P, P]
    L.wo_centrality.restype = I32
    L.wo_centrality.argtypes = [P, I, I, P, U64, P, P]
    if hasattr(L, "wo_eigen"):
        L.wo_eigen.restype = I32
        L.wo_eigen.argtypes = [P, I, I, I, I, D, U64, U64, P, P, P, P]
    L.wo_pagerank_adjoint.restype = I32
    L.wo_pagerank_adjoint.argtypes = [P, D, I, D, U32, P, P, U32, D, P, P, P]
    L.wc_graph_rmat.restype = I32
    L.wc_graph_rmat.argtypes = [U32, U32, D, D, D, U64, I32, C.POINTER(HostCsr)]
    L.wc_graph_gnm.restype = I32
    L.wc_graph_gnm.argtypes = [U64, U64, U64, I32, C.POINTER(HostCsr)]
    L.wc_host_csr_free.argtypes = [C.POINTER(HostCsr)]


class HostCsr(C.Structure):
    """wc_host_csr (include/warren_cuda.h): a generated graph's CSR."""

    _fields_ = [("id_space", U64), ("edges", U64), ("offsets", C.POINTER(U64)),
                ("targets", C.POINTER(U32)), ("external_ids", C.POINTER(C.c_int64))]


class SyntheticGraph:
    """A generated graph's CSR arrays (offsets u64, targets u32)."""

    def __init__(self, offsets, targets):
        self.offsets = offsets
        self.targets = targets
        self.id_space = len(offsets) - 1
        self.edges = len(targets)


def _take(csr):
    n, m = csr.id_space, csr.edges
    off = np.ctypeslib.as_array(csr.offsets, shape=(n + 1,)).copy()
    tgt = np.ctypeslib.as_array(csr.targets, shape=(max(m, 1),))[:m].copy()
    lib().wc_host_csr_free(C.byref(csr))
    return SyntheticGraph(off, tgt)


def rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, undirected=False):
    """The benchmark's seeded R-MAT graph (the generator the CUDA library
    also exports, compiled here from the same source)."""
    csr = HostCsr()
    _check(lib().wc_graph_rmat(scale, edge_factor, a, b, c, seed, int(undirected), C.byref(csr)))
    return _take(csr)


def gnm(n, m, seed=1, undirected=False):
    """The benchmark's seeded G(n, m) graph, as rmat."""
    csr = HostCsr()
    _check(lib().wc_graph_gnm(n, m, seed, int(undirected), C.byref(csr)))
    return _take(csr)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(P)


class OracleError(RuntimeError):
    def __init__(self, status):
        super().__init__(f"oracle status {status}")
        self.status = status


def _check(status):
    if status != OK:
        raise OracleError(status)


def set_threads(n: int) -> None:
    lib().wo_set_threads(n)


def set_chunk(n: int) -> None:
    """The reduction chunk (compute/reduce.rs:20): 65536, or 4 under test."""
    lib().wo_set_chunk(n)


class Graph:
    """A built graph: forward CSR, and the reverse CSR if `reverse`."""

    def __init__(self, handle, n, reverse):
        self.handle = handle
        self.n = n
        self.reverse = reverse
        self.m = lib().wo_graph_edges(handle)
        self.weighted = bool(lib().wo_graph_weighted(handle))

    @classmethod
    def from_edges(cls, n, edges, weighted, reverse=True, relations=1):
        """`edges`: (relation, source, target, weight) as the reference's
        test fixtures list them (compute/reference.rs:6-47)."""
        e = np.array(edges, dtype=np.float64).reshape(-1, 4)
        rel = np.ascontiguousarray(e[:, 0].astype(np.uint32))
        src = np.ascontiguousarray(e[:, 1].astype(np.uint64))
        dst = np.ascontiguousarray(e[:, 2].astype(np.uint64))
        w = np.ascontiguousarray(e[:, 3]) if weighted else None
        h = lib().wo_graph_build(n, relations, len(e), _ptr(rel), _ptr(src), _ptr(dst), _ptr(w),
                                 1 if reverse else 0)
        return cls(h, n, reverse)

    @classmethod
    def from_csr(cls, n, offsets, targets, weights=None, reverse=True):
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        targets = np.ascontiguousarray(targets, dtype=np.uint32)
        if weights is not None:
            weights = np.ascontiguousarray(weights, dtype=np.float64)
        h = lib().wo_graph_from_csr(n, len(targets), _ptr(offsets), _ptr(targets), _ptr(weights),
                                    1 if reverse else 0)
        return cls(h, n, reverse)

    def csr(self):
        off = np.zeros(self.n + 1, np.uint64)
        tgt = np.zeros(self.m, np.uint32)
        w = np.zeros(self.m, np.float64) if self.weighted else None
        roff = np.zeros(self.n + 1, np.uint64) if self.reverse else None
        rtgt = np.zeros(self.m, np.uint32) if self.reverse else None
        rw = np.zeros(self.m, np.float64) if (self.reverse and self.weighted) else None
        lib().wo_graph_copy(self.handle, _ptr(off), _ptr(tgt), _ptr(w), _ptr(roff), _ptr(rtgt),
                            _ptr(rw))
        return off, tgt, w, roff, rtgt, rw

    def __del__(self):
        if getattr(self, "handle", None):
            try:
                lib().wo_graph_free(self.handle)
            except Exception:
                pass
            self.handle = None


DTYPES = {1: np.float64, 0: np.float32, 2: np.int64, 3: np.uint8}


def product(g, semiring, x, y, transpose=False, weighted=-1, mask=None, mask_dtype=1,
            complement=False, replace=False, accumulate=-1, force_push=False):
    """compute/product/mod.rs:77-110; `y` is updated in place; returns status."""
    dtype = {np.float64: 1, np.float32: 0, np.int64: 2, np.uint8: 3, np.bool_: 3}[y.dtype.type]
    width = 1 if x.ndim == 1 else x.shape[1]
    return lib().wo_product(g.handle, semiring, int(transpose), weighted, _ptr(mask), mask_dtype,
                            int(complement), int(replace), accumulate, dtype, width, _ptr(x),
                            _ptr(y), int(force_push))


def pagerank(g, damping=0.85, tol=1e-6, max_iter=100, tombstones=None, seed=None, weighted=-1):
    """compute/pagerank/mod.rs:96-151: returns (ranks, iterations, delta, threshold)."""
    ranks = np.zeros(g.n, np.float64)
    it = np.zeros(1, np.uint32)
    delta = np.zeros(1, np.float64)
    thr = np.zeros(1, np.float64)
    has_tol = tol is not None
    st = lib().wo_pagerank(g.handle, _ptr(tombstones), damping, int(has_tol),
                           float(tol) if has_tol else 0.0, weighted, max_iter, _ptr(seed),
                           _ptr(ranks), _ptr(it), _ptr(delta), _ptr(thr))
    _check(st)
    return ranks, int(it[0]), float(delta[0]), float(thr[0])


def tombstone_words(n, ids):
    words = np.zeros((n + 63) // 64, np.uint64)
    for i in ids:
        words[i // 64] |= np.uint64(1) << np.uint64(i % 64)
    return words


def bfs(g, starts, direction=0, max_depth=None, max_results=None, filter_ids=None,
        pulling=False):
    """traversal/bfs.rs:34-45: ([(node, depth, via)], stats dict).  With
    `pulling`, levels may be pulled as reachable_set's are (level.rs:184-284),
    the result limit applying to them too."""
    starts = np.ascontiguousarray(starts, dtype=np.uint64)
    cap = g.n + 1
    visits = np.zeros(3 * cap, np.uint64)
    count = np.zeros(1, np.uint64)
    stats = np.zeros(5, np.uint64)
    filt = tombstone_words(g.n, filter_ids) if filter_ids is not None else None
    st = lib().wo_level_search(g.handle, direction, _ptr(starts), len(starts),
                               0xFFFFFFFF if max_depth is None else max_depth,
                               0xFFFFFFFFFFFFFFFF if max_results is None else max_results,
                               _ptr(filt), 1 if pulling else 0, _ptr(visits), cap, _ptr(count),
                               _ptr(stats))
    _check(st)
    c = int(count[0])
    v = visits[: 3 * c].reshape(-1, 3)
    out = [(int(a), int(b), None if int(cv) == 0xFFFFFFFFFFFFFFFF else int(cv)) for a, b, cv in v]
    return out, _stats(stats)


def _stats(s):
    return {"nodes_visited": int(s[0]), "edges_traversed": int(s[1]), "truncated": bool(s[2]),
            "levels": int(s[3]), "pulled_levels": int(s[4])}


def reachable_set(g, starts, direction=0, max_depth=None):
    starts = np.ascontiguousarray(starts, dtype=np.uint64)
    nodes = np.zeros(g.n + 1, np.uint64)
    count = np.zeros(1, np.uint64)
    stats = np.zeros(5, np.uint64)
    st = lib().wo_reachable_set(g.handle, direction, _ptr(starts), len(starts),
                                0xFFFFFFFF if max_depth is None else max_depth, _ptr(nodes),
                                len(nodes), _ptr(count), _ptr(stats))
    _check(st)
    return [int(v) for v in nodes[: int(count[0])]], _stats(stats)


def bfs_depths(g, sources, caps):
    """Per-source plain BFS depths (255: not reached) and edges_traversed."""
    sources = np.ascontiguousarray(sources, dtype=np.uint64)
    caps = np.ascontiguousarray(caps, dtype=np.uint32)
    out = np.zeros((len(sources), g.n), np.uint8)
    edges = np.zeros(len(sources), np.uint64)
    _check(lib().wo_bfs_depths(g.handle, _ptr(sources), _ptr(caps), len(sources), _ptr(out),
                               _ptr(edges)))
    return out, edges


def bfs_depths_batched64(g, sources, caps):
    """bfs_depths by the reference's own batched shape (multi_source.rs:
    64 sources a word, atomic-OR push, per-level settle): same results."""
    sources = np.ascontiguousarray(sources, dtype=np.uint64)
    caps = np.ascontiguousarray(caps, dtype=np.uint32)
    out = np.zeros((len(sources), g.n), np.uint8)
    edges = np.zeros(len(sources), np.uint64)
    _check(lib().wo_bfs_depths_batched64(g.handle, _ptr(sources), _ptr(caps), len(sources),
                                         _ptr(out), _ptr(edges)))
    return out, edges


def sssp_i64(g, sources, max_iter):
    """compute_sql/library/sssp_vector.sql:14-66 over i64, per source."""
    sources = np.ascontiguousarray(sources, dtype=np.uint64)
    max_iter = np.ascontiguousarray(max_iter, dtype=np.uint32)
    out = np.zeros((len(sources), g.n), np.int64)
    its = np.zeros(len(sources), np.uint32)
    _check(lib().wo_sssp_i64(g.handle, _ptr(sources), _ptr(max_iter), len(sources), _ptr(out),
                             _ptr(its)))
    return out, its


def components(g):
    """traversal/components.rs:21-58: (labels u64[n], nodes_visited,
    edges_traversed)."""
    labels = np.zeros(g.n, np.uint64)
    nv = np.zeros(1, np.uint64)
    et = np.zeros(1, np.uint64)
    _check(lib().wo_components(g.handle, _ptr(labels), _ptr(nv), _ptr(et)))
    return labels, int(nv[0]), int(et[0])


REDUCTIONS = ["sum", "max", "min", "l1", "l2", "nnz"]
NORMS = ["l1", "l2", "linf"]
_DT = {np.dtype(np.float32): 0, np.dtype(np.float64): 1, np.dtype(np.int64): 2,
       np.dtype(np.bool_): 3, np.dtype(np.uint8): 3}


def reduce(x, reduction, width=1, tombstones=None):
    """compute/reduce.rs:118-153: the reduction of x's elements (rows of
    `width`), skipping tombstoned rows; None for the max / min of none."""
    x = np.ascontiguousarray(x)
    out = np.zeros(1, np.float64)
    null = np.zeros(1, np.int32)
    _check(lib().wo_reduce(_DT[x.dtype], _ptr(x), x.size // width, width, _ptr(tombstones),
                           REDUCTIONS.index(reduction), _ptr(out), _ptr(null)))
    return None if null[0] else float(out[0])


def norm_diff(a, b, norm, width=1):
    """compute/reduce.rs:175-206."""
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    out = np.zeros(1, np.float64)
    _check(lib().wo_norm_diff(_DT[a.dtype], _ptr(a), a.size // width, _DT[b.dtype], _ptr(b),
                              b.size // width, width, NORMS.index(norm), _ptr(out)))
    return float(out[0])


def sample_sources(n, tombstones=None, population=None, complement=False, k=None, seed=0):
    """centrality/sources.rs:55-123: the chosen sources, ascending."""
    pop = None if population is None else np.ascontiguousarray(np.asarray(population) != 0,
                                                                dtype=np.uint8)
    out = np.zeros(max(n, 1), np.uint64)
    count = np.zeros(1, np.uint64)
    _check(lib().wo_sample_sources(n, _ptr(tombstones), _ptr(pop), int(complement),
                                   -1 if k is None else int(k), seed & (2**64 - 1), _ptr(out),
                                   _ptr(count)))
    return out[:int(count[0])].copy()


def betweenness(g, sources, tombstones=None, normalized=True, endpoints=False, directed=True):
    """betweenness.rs with paths.rs (unweighted), sources in order: f64[n]."""
    src = np.ascontiguousarray(sources, dtype=np.uint64)
    out = np.zeros(g.n, np.float64)
    _check(lib().wo_betweenness(g.handle, _ptr(src), len(src), _ptr(tombstones), int(normalized),
                                int(endpoints), int(directed), _ptr(out)))
    return out


def centrality(g, measure, sources, tombstones=None, wf_improved=True):
    """closeness.rs (measure "closeness" or "harmonic") from `sources`
    (ascending), the batched measures' order: f64[n]."""
    src = np.ascontiguousarray(sources, dtype=np.uint64)
    out = np.zeros(g.n, np.float64)
    _check(lib().wo_centrality(g.handle, 0 if measure == "closeness" else 1, int(wf_improved),
                               _ptr(src), len(src), _ptr(tombstones), _ptr(out)))
    return out


def topk(x, k, descending=True, tombstones=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    nodes = np.zeros(max(k, 1), np.uint64)
    vals = np.zeros(max(k, 1), np.float64)
    count = np.zeros(1, np.uint64)
    _check(lib().wo_topk_f64(_ptr(x), len(x), _ptr(tombstones), k, int(descending), _ptr(nodes),
                             _ptr(vals), _ptr(count)))
    c = int(count[0])
    return nodes[:c].copy(), vals[:c].copy()


def uniform(seed, stream, node):
    return lib().wo_uniform(seed, stream, node)


def float_op(op, a, b):
    """map/arithmetic.rs:49-79: (status, value); op 0..3 = + − × ÷."""
    out = D(0.0)
    st = lib().wo_float(op, a, b, C.byref(out))
    return st, out.value


def pagerank_adjoint(g, loss_targets, damping=0.85, tol=1e-10, max_iter=100, adjoint_tol=1e-14):
    """The FP64 CPU adjoint: (grad[losses, edges], ranks, (forward, adjoint) iterations)."""
    offs = np.zeros(len(loss_targets) + 1, np.uint64)
    for i, t in enumerate(loss_targets):
        offs[i + 1] = offs[i] + len(t)
    nodes = np.ascontiguousarray(np.concatenate([np.asarray(t, np.uint64) for t in loss_targets]))
    grad = np.zeros((len(loss_targets), g.m), np.float64)
    ranks = np.zeros(g.n, np.float64)
    its = np.zeros(2, np.uint32)
    _check(lib().wo_pagerank_adjoint(g.handle, damping, int(tol is not None),
                                     0.0 if tol is None else tol, max_iter, _ptr(nodes),
                                     _ptr(offs), len(loss_targets), adjoint_tol, _ptr(grad),
                                     _ptr(ranks), _ptr(its)))
    return grad, ranks, its
