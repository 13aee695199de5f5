// pagerank.h — the state of one PageRank solve on the device, shared by
// wc_pagerank, the batched personalised PageRank and the adjoint.
#pragma once

#include "product.h"
#include "runtime.cuh"

namespace wc {

struct PrState {
  uint32_t n;
  double* x[2];
  double* msg[2];
  const double* out;
  const double* shares;  // NULL: uniform, `start` at every live row
  const uint64_t* tomb;
  double start, damping, teleport, threshold;
  bool has_tol;
  double* delta;     // per iteration
  double* dangling;  // per iteration (+1)
  double* partials;  // 2 per block
  unsigned* counter;
  uint32_t* iterations;
  int32_t* done;
  const int32_t* cancel;
  uint32_t* pace;  // host-mapped: [0] iterations done, [1] stopped
  DeviceError* err;
};

struct PageRankRun {
  wc_pagerank_opts opts;
  uint64_t live = 0;
  double nodes = 0.0;
  uint32_t grid = 1;
  uint32_t long_grid = 1;  // pr_long_kernel's blocks (locality order)
  // The solve pulls over the version's locality-ordered CSC (v->loc), its
  // vectors in that numbering; inputs are renumbered in by setup and the
  // ranks out by result.  Off for callers that read the vectors themselves.
  bool local = false;
  DevBuf *x = nullptr, *msg = nullptr, *out = nullptr, *shares = nullptr, *tomb = nullptr,
         *scalars = nullptr;
  PrState s;

  wc_status setup(Ctx& ctx, const wc_pagerank_opts* o, const uint64_t* tomb_host,
                  const double* seed, bool in_locality_order = false);
  // The CSC the iterations pull over and the grid for it.
  const DevCsr& csc(const wc_version* v) const { return local ? v->loc.csc : v->rev; }
  wc_status run(Ctx& ctx);
  wc_status result(Ctx& ctx, double* ranks, uint32_t* iterations, double* margin);
};

// Over the locality-ordered CSC, the messages of the nodes numbered below
// this (the most gathered) are kept in L1: 64 KB of them, what the SM's L1
// holds beside four blocks' staging rings.
constexpr uint32_t kPageRankHotNodes = 8192;

uint64_t live_count(const uint64_t* tomb, uint64_t n);
// pr_init_kernel: the start vector, its messages and dangling rank.
wc_status launch_pr_init(const PrState& s, uint32_t grid, cudaStream_t stream);
// One iteration (pr_iter_kernel) over L's units.
struct PullLaunch;
wc_status launch_part_iteration(const PullLaunch& L, const PrState& s, uint32_t it,
                                uint32_t blocks);
// Drops a version's partitioned solve (wc_pagerank_part_*) when it is released.
void pagerank_part_forget(const wc_version* v);
// The row-partitioned search's and product's state kept with a version
// (bfs_part.cu), dropped when the version is released.
void bfs_part_forget(const wc_version* v);
// Blocks of an iteration launch over `csc`; of the long-row pass that
// follows it in the locality order; and the block sums the step keeps.
uint32_t pagerank_grid(const DevCsr& csc);
uint32_t pagerank_long_grid(const DevCsr& csc);
uint32_t pagerank_partial_blocks(const DevCsr& csc);

}  // namespace wc
