"""pg_warren_b200 — the B200 (sm_100a) backend of pg_warren's whole-graph
compute path, behind the C ABI of include/warren_cuda.h.

``api`` mirrors warren-core's compute interface (spmv / spmm / pagerank /
bfs / reachable_set / eigen / top_k) over the CUDA library; ``build``
compiles it.  Importing the package does not load the library; the first
call does, and fails loudly if it was not built.
"""

from .api import *  # noqa: F401,F403
from .api import (Budget, GraphVersion, Product, PageRank, Limits, EigenOptions, Interrupts,
                  spmv, spmm, pagerank, pagerank_noalloc, bfs, bfs_depths, reachable_set, reachable, components, bfs_batched,
                  minplus_batched, ppr_batched, autotune, set_schedule, eigen, pagerank_adjoint, top_k, rmat, gnm,
                  edge_weights, node_set, HostGraph, Sampling, Centrality, sample_sources,
                  closeness_centrality, harmonic_centrality, vector_reduce, vector_norm_diff,
                  vector_map, betweenness_centrality)
from ._abi import load, LIBRARY

__all__ = ["Budget", "GraphVersion", "Product", "PageRank", "Limits", "EigenOptions",
           "Interrupts", "spmv", "spmm", "pagerank", "pagerank_noalloc", "bfs", "bfs_depths", "reachable_set",
           "reachable", "components", "bfs_batched", "minplus_batched", "ppr_batched", "autotune", "set_schedule", "eigen",
           "pagerank_adjoint", "top_k", "rmat", "gnm", "edge_weights", "node_set", "HostGraph",
           "Sampling", "Centrality", "sample_sources", "closeness_centrality",
           "harmonic_centrality", "vector_reduce", "vector_norm_diff", "vector_map",
           "betweenness_centrality",
           "load", "LIBRARY"]
