// bfs.h — one level-synchronous search on the device (traversal/level.rs).
#pragma once

#include <map>
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

// The device side of one level, indexed by the level within the chunk the
// host queued: what the level's kernels read (its frontier and the switch's
// choice) and what they add up for the next level.
struct LevelState {
  uint32_t count;                 // frontier nodes
  uint32_t pull;                  // the level pulls
  unsigned long long mf;          // Σ row length (search direction) of the frontier
  unsigned long long visited_rdeg;  // Σ opposite-direction row length of the visited nodes
  // Added up by the level's kernels:
  unsigned long long next_deg;    // Σ row length (search direction) over nodes admitted
  unsigned long long next_rdeg;   // Σ row length (opposite direction) over nodes admitted
  unsigned long long edges;       // row entries scanned by a pulled level
  uint32_t next_count;
  uint32_t big_count;             // frontier rows deferred to push_big_kernel
  uint32_t huge_count;            // of which pushed by the whole grid (listed from the end)
  uint32_t done;                  // push_big_kernel's blocks finished
};

// The switch (level.rs:19-29, 184-211 for the reference's; a GPU-tuned one
// for bfs), evaluated where the level is planned.
struct SwitchArgs {
  uint32_t rule;  // SwitchRule
  uint32_t reverse_allowed;
  uint64_t n;
  uint64_t total_rdeg;
};

// A search is started (starts checked and admitted, buffers set up), then
// advanced level by level.  Its buffers come from the version's scratch
// pool for the length of one call, or from `owned` for a search that lives
// across calls (a cursor).
struct Search {
  int direction = WC_OUT;
  bool reverse_allowed = false;             // may a level be pulled (reachable_set)
  bool ordering_by_node_in_pulled = false;  // pulled levels list nodes ascending
  DevBuf *depth = nullptr, *via = nullptr, *queue[2] = {nullptr, nullptr}, *fbits = nullptr,
         *counters = nullptr, *filter = nullptr, *big = nullptr;
  std::map<int, DevBuf>* owned = nullptr;   // buffers by pool tag, if not the pool's
  // The per-node depths and vias the search writes: the caller's device
  // arrays when set before start(), else the search's own buffers.
  uint32_t* depth_p = nullptr;
  unsigned long long* via_p = nullptr;
  std::vector<uint32_t> seeds;
  std::vector<Level> levels;
  wc_traversal_stats stats{};
  // Where the search stands between advances.
  uint32_t depth_reached = 0;  // levels expanded so far
  uint32_t max_depth = 0;
  SwitchArgs sw{};
  LevelState next_plan{};      // the plan of the next level (count 0: exhausted)
  uint32_t last_admitted = 0;  // nodes admitted by the last level expanded
  bool init_pending = false;   // the device state is set up with the first levels
  uint32_t pending_chunk = 0;  // levels of a deferred chunk not yet read back

  wc_status run(Ctx& ctx, int direction, const uint64_t* starts, uint64_t start_count,
                uint32_t max_depth, const uint64_t* filter, SwitchRule rule);
  wc_status start(Ctx& ctx, int direction, const uint64_t* starts, uint64_t start_count,
                  uint32_t max_depth, const uint64_t* filter, SwitchRule rule);
  // Expands up to `max_levels` more levels (fewer once the frontier empties
  // or the depth cap is met).  With `defer_last` the last chunk the cap
  // allows is queued without waiting for it: the caller waits (after
  // queueing its own work) and then calls collect() for the stats.
  wc_status advance(Ctx& ctx, uint32_t max_levels, bool defer_last = false);
  void collect(Ctx& ctx);
  bool exhausted() const { return next_plan.count == 0; }
  wc_status ordered(Ctx& ctx, std::vector<uint64_t>& rows, bool with_via);

 private:
  wc_status buffer(Ctx& ctx, int tag, uint64_t bytes, DevBuf** out);
  wc_status enqueue_init(Ctx& ctx, bool staged);
  bool absorb(const LevelState* plan, uint32_t chunk);
};

}  // namespace wc
