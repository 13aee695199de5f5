"""ctypes declarations of include/warren_cuda.h.

The library is the in-tree ``libwarren_cuda.so``; loading fails loudly when
it is missing (there is no CPU fallback: a caller without the library keeps
its native kernels).
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libwarren_cuda.so")

P = C.c_void_p
U64 = C.c_uint64
U32 = C.c_uint32
I32 = C.c_int32
D = C.c_double

# enums (include/warren_cuda.h)
F32, F64, I64, BOOL = 0, 1, 2, 3
OUT, IN, BOTH = 0, 1, 2
OP_NONE = -1
SEMIRINGS = ["plus_times", "min_plus", "max_plus", "max_times", "min_times", "lor_land",
             "any_pair", "plus_pair", "plus_first", "plus_second", "min_first", "min_second",
             "max_second"]
BINARY_OPS = ["first", "second", "pair", "plus", "times", "min", "max", "lor", "land", "any"]
UNREACHED = 0xFFFFFFFF
NO_VIA = 0xFFFFFFFFFFFFFFFF


class ErrorDetail(C.Structure):
    _fields_ = [("requested", U64), ("in_use", U64), ("limit", U64), ("node", U64),
                ("expected", U64), ("found", U64), ("degree", D), ("cuda_error", I32),
                ("message", C.c_char * 200)]


PROGRESS_FN = C.CFUNCTYPE(None, P, C.c_char_p, U64, U64)


class Call(C.Structure):
    _fields_ = [("memory", P), ("cancel", C.POINTER(I32)), ("progress", PROGRESS_FN),
                ("progress_context", P), ("stream", P), ("flags", U32), ("timeout_ms", U32),
                ("detail", C.POINTER(ErrorDetail))]


class CsrHost(C.Structure):
    _fields_ = [("id_space", U64), ("edges", U64), ("offsets", P), ("targets", P),
                ("weights", P), ("reverse_offsets", P), ("reverse_targets", P),
                ("reverse_weights", P), ("reverse_on_device", I32)]


class VersionInfo(C.Structure):
    _fields_ = [("id_space", U64), ("edges", U64), ("device_bytes", U64), ("weighted", I32),
                ("integral_weights", I32), ("device", I32), ("symmetric", I32),
                ("scratch_bytes", U64)]


class Mask(C.Structure):
    _fields_ = [("values", P), ("dtype", I32), ("complement", I32)]


class ProductC(C.Structure):
    _fields_ = [("semiring", I32), ("transpose", I32), ("weighted", I32),
                ("mask", C.POINTER(Mask)), ("replace", I32), ("accumulate", I32)]


class PageRankOpts(C.Structure):
    _fields_ = [("damping", D), ("tol", D), ("has_tol", I32), ("weighted", I32),
                ("max_iter", U32), ("seed", P)]


class TraversalStats(C.Structure):
    _fields_ = [("nodes_visited", U64), ("edges_traversed", U64), ("truncated", I32),
                ("levels", U32), ("pulled_levels", U32)]


class Limits(C.Structure):
    _fields_ = [("max_depth", U32), ("max_results", U64)]


class Schedule(C.Structure):
    _fields_ = [("columns_per_pass", U32), ("rows_per_unit", U32), ("blocks_per_sm", U32),
                ("reserved", U32)]


class BetweennessOpts(C.Structure):
    _fields_ = [("normalized", I32), ("endpoints", I32), ("directed", I32),
                ("blocks_per_sm", U32)]


class CentralityOpts(C.Structure):
    _fields_ = [("measure", U32), ("wf_improved", U32), ("columns_per_pass", U32),
                ("blocks_per_sm", U32)]


class EigenOpts(C.Structure):
    _fields_ = [("k", U32), ("which", I32), ("op", I32), ("symmetrize", I32), ("weighted", I32),
                ("tol", D), ("max_iter", U64), ("seed", U64)]


class EigenStats(C.Structure):
    _fields_ = [("iterations", U64), ("components", U64), ("exact", U32), ("converged", I32)]


class PageRankPartInfo(C.Structure):
    _fields_ = [("row_begin", U64), ("row_end", U64), ("id_space", U64), ("live", U64),
                ("dangling", D), ("threshold", D)]


class BfsPartInfo(C.Structure):
    _fields_ = [("row_begin", U64), ("row_end", U64), ("id_space", U64), ("words", U64),
                ("frontier", U64), ("frontier_edges", U64)]


class HostCsr(C.Structure):
    _fields_ = [("id_space", U64), ("edges", U64), ("offsets", C.POINTER(U64)),
                ("targets", C.POINTER(U32)), ("external_ids", C.POINTER(C.c_int64))]


# (name, restype, argtypes) of every entry point the header declares.
SIGNATURES = [
    ("wc_status_name", C.c_char_p, [I32]),
    ("wc_budget_create", I32, [U64, C.POINTER(P)]),
    ("wc_budget_destroy", None, [P]),
    ("wc_budget_in_use", U64, [P]),
    ("wc_budget_peak", U64, [P]),
    ("wc_version_upload", I32, [U64, U64, C.POINTER(CsrHost), P, C.POINTER(Call), C.POINTER(P)]),
    ("wc_version_load_segments", I32, [U64, U64, U64, P, U64, P, U64, P, U64, P, U64, I32, P,
                                       C.POINTER(Call), C.POINTER(P)]),
    ("wc_version_release", I32, [P]),
    ("wc_version_info_get", I32, [P, C.POINTER(VersionInfo)]),
    ("wc_version_sync", I32, [P, C.POINTER(Call)]),
    ("wc_serves", I32, [C.c_char_p, I32]),
    ("wc_kernel_launches", U64, []),
    ("wc_version_timing", D, [P, C.c_char_p, C.POINTER(U32)]),
    ("wc_random_uniform", I32, [P, C.POINTER(Call), U64, U64, P]),
    ("wc_selftest_bounded_wait", I32, [C.POINTER(Call), U32]),
    ("wc_spmv", I32, [P, C.POINTER(Call), C.POINTER(ProductC), I32, P, P]),
    ("wc_spmm", I32, [P, C.POINTER(Call), C.POINTER(ProductC), I32, U32, P, P]),
    ("wc_pagerank", I32, [P, C.POINTER(Call), C.POINTER(PageRankOpts), P, P, C.POINTER(U32)]),
    ("wc_pagerank_noalloc", I32, [P, C.POINTER(Call), C.POINTER(PageRankOpts), P, P,
                             C.POINTER(U32)]),
    ("wc_pagerank_last_margin", D, [P]),
    ("wc_pagerank_part_rows", I32, [P, U32, P]),
    ("wc_pagerank_part_begin", I32, [P, C.POINTER(Call), C.POINTER(PageRankOpts), P, U32, U32,
                                     P, P, C.POINTER(PageRankPartInfo)]),
    ("wc_pagerank_part_step", I32, [P, C.POINTER(Call), U32, D, C.POINTER(D)]),
    ("wc_pagerank_part_end", I32, [P, C.POINTER(Call), U32, P]),
    ("wc_spmv_part_rows", I32, [P, I32, U32, P]),
    ("wc_spmv_part", I32, [P, C.POINTER(Call), C.POINTER(ProductC), I32, U32, U32, P, P]),
    ("wc_bfs_part_rows", I32, [P, I32, U32, P]),
    ("wc_bfs_part_begin", I32, [P, C.POINTER(Call), I32, P, U64, U32, U32, U32, P,
                                C.POINTER(BfsPartInfo)]),
    ("wc_bfs_part_step", I32, [P, C.POINTER(Call), U32, U64, P]),
    ("wc_bfs_part_end", I32, [P, C.POINTER(Call), P]),
    ("wc_bfs", I32, [P, C.POINTER(Call), I32, P, U64, C.POINTER(Limits), P, P, P,
                     C.POINTER(TraversalStats)]),
    ("wc_bfs_visits", I32, [P, C.POINTER(Call), I32, P, U64, C.POINTER(Limits), P, P, U64,
                            C.POINTER(U64), C.POINTER(TraversalStats)]),
    ("wc_reachable_set", I32, [P, C.POINTER(Call), I32, P, U64, U32, P, U64, C.POINTER(U64),
                               C.POINTER(TraversalStats)]),
    ("wc_bfs_cursor_open", I32, [P, C.POINTER(Call), I32, P, U64, C.POINTER(Limits), P, I32,
                                 C.POINTER(P)]),
    ("wc_bfs_cursor_next", I32, [P, C.POINTER(Call), C.POINTER(U64), C.POINTER(I32)]),
    ("wc_bfs_cursor_read", I32, [P, U64, U64, P]),
    ("wc_bfs_cursor_stop", I32, [P, C.POINTER(Call), U64]),
    ("wc_bfs_cursor_stats", I32, [P, C.POINTER(TraversalStats)]),
    ("wc_bfs_cursor_destroy", None, [P]),
    ("wc_reachable", I32, [P, C.POINTER(Call), I32, U64, U64, U32, C.POINTER(I32),
                           C.POINTER(TraversalStats)]),
    ("wc_components", I32, [P, C.POINTER(Call), P, C.POINTER(TraversalStats)]),
    ("wc_autotune", I32, [P, C.POINTER(Call), I32, U32, C.POINTER(Schedule)]),
    ("wc_schedule_set", I32, [P, I32, U32, C.POINTER(Schedule)]),
    ("wc_bfs_batched", I32, [P, C.POINTER(Call), P, P, U32, P, P]),
    ("wc_minplus_batched", I32, [P, C.POINTER(Call), P, P, U32, P, P]),
    ("wc_ppr_batched", I32, [P, C.POINTER(Call), C.POINTER(PageRankOpts), P, P, U32, P, P]),
    ("wc_sample_sources", I32, [U64, P, P, I32, C.c_int64, U64, P, C.POINTER(U64)]),
    ("wc_betweenness", I32, [P, C.POINTER(Call), C.POINTER(BetweennessOpts), P, U64, P, P]),
    ("wc_centrality", I32, [P, C.POINTER(Call), C.POINTER(CentralityOpts), P, U64, P, P]),
    ("wc_eigen", I32, [P, C.POINTER(Call), C.POINTER(EigenOpts), P, P, P, C.POINTER(EigenStats)]),
    ("wc_pagerank_adjoint", I32, [P, C.POINTER(Call), C.POINTER(PageRankOpts), P, P, U32, D, P,
                                  P, P]),
    ("wc_vector_map", I32, [P, C.POINTER(Call), P, U32, P, U32, U32, P, P, P, P, U32, P,
                            C.POINTER(U32)]),
    ("wc_vector_reduce", I32, [P, C.POINTER(Call), I32, P, U32, P, I32, C.POINTER(D),
                               C.POINTER(I32)]),
    ("wc_vector_norm_diff", I32, [P, C.POINTER(Call), I32, P, U64, I32, P, U64, U32, I32,
                                  C.POINTER(D)]),
    ("wc_topk", I32, [P, C.POINTER(Call), I32, P, P, U64, I32, P, P, C.POINTER(U64)]),
    ("wc_graph_rmat", I32, [U32, U32, D, D, D, U64, I32, C.POINTER(HostCsr)]),
    ("wc_graph_gnm", I32, [U64, U64, U64, I32, C.POINTER(HostCsr)]),
    ("wc_host_csr_free", None, [C.POINTER(HostCsr)]),
    ("wc_host_transpose", I32, [U64, U64, P, P, P, P, P, P]),
]

_lib = None


def load() -> C.CDLL:
    """The library, declared; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise ImportError(
                f"{LIBRARY} is missing: build it with `python -m pg_warren_b200.build` "
                "(there is no CPU fallback)")
        lib = C.CDLL(LIBRARY)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
