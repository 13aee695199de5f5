// batched.h — buffers and entry points shared by the batched searches.
#pragma once

#include <vector>

#include "runtime.cuh"

namespace wc {

struct BatchBuffers {
  DevBuf *V = nullptr, *F = nullptr, *bits = nullptr, *masks = nullptr, *counts = nullptr,
         *nacc = nullptr, *acc = nullptr, *touched = nullptr;
  DevBuf* pulled = nullptr;  // u32: levels that pulled, in a timed call
  wc_status reserve(Ctx& ctx, uint32_t words, uint32_t levels);
};

// A centrality pass's per-node totals (kept across passes) and its flag
// for a frontier left after the last level.
struct CentArgs {
  unsigned long long* reached;  // sources (other than the node) that reach it
  unsigned long long* dsum;     // their summed distances
  double* harm;                 // Σ 1 / distance, batch by batch
  int* cut;
  bool keep_only = false;       // keep the snapshots for the caller's kernels, count nothing
};

wc_schedule default_bfs_schedule(uint32_t width);
// One batched BFS pass of up to `columns` (64 .. 1024) sources, every cap
// `levels`, whose per-node counts go to `cent` instead of depths.
wc_status bfs_centrality_pass(Ctx& ctx, BatchBuffers& b, uint32_t columns,
                              const uint64_t* sources_dev, const uint32_t* caps_dev, uint32_t k,
                              uint32_t levels, uint32_t blocks_per_sm, const CentArgs& cent);
wc_status bfs_batched_run(Ctx& ctx, const wc_schedule& sched, const uint64_t* sources_dev,
                          const uint32_t* caps_dev, const uint32_t* caps_host, uint32_t width,
                          uint8_t* depth_dev, unsigned long long* edges_dev);

// The 32-bit batched min-plus (batched_minplus32.cu): a pass of up to 64
// columns, sources / caps / the call's column of each in device memory.
typedef wc_status (*Mp32Fn)(Ctx&, const uint64_t*, const uint32_t*, const uint32_t*, uint32_t,
                            uint32_t, int64_t*, uint32_t*, uint32_t);
Mp32Fn mp32_for(uint32_t columns);
wc_status mp32_reserve(Ctx& ctx, uint32_t columns);

// `count` seeded node ids below n, for the tuners' sample columns.
void sample_nodes(uint32_t n, uint32_t count, std::vector<uint64_t>& out, uint64_t salt);

}  // namespace wc
