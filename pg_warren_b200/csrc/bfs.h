// bfs.h — one level-synchronous search on the device (traversal/level.rs).
#pragma once

#include <vector>

#include "runtime.cuh"

namespace wc {

enum SwitchRule { REFERENCE_SWITCH = 0, GPU_SWITCH = 1 };

struct Level {
  bool pulled;
  uint32_t frontier;
  uint64_t frontier_entries;  // Σ row length of the frontier (what a push scans)
  uint64_t scanned;           // row entries scanned (a pull stops at its first hit)
  uint32_t admitted;
};

struct Search {
  int direction = WC_OUT;
  bool reverse_allowed = false;             // may a level be pulled (reachable_set)
  bool ordering_by_node_in_pulled = false;  // pulled levels list nodes ascending
  DevBuf *depth = nullptr, *via = nullptr, *queue[2] = {nullptr, nullptr}, *fbits = nullptr,
         *counters = nullptr, *filter = nullptr, *big = nullptr;
  std::vector<uint32_t> seeds;
  std::vector<Level> levels;
  wc_traversal_stats stats{};

  wc_status run(Ctx& ctx, int direction, const uint64_t* starts, uint64_t start_count,
                uint32_t max_depth, const uint64_t* filter, SwitchRule rule);
  wc_status ordered(Ctx& ctx, std::vector<uint64_t>& rows, bool with_via);
};

}  // namespace wc
