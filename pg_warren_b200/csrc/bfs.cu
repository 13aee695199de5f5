// bfs.cu — wc_bfs, wc_bfs_visits, wc_reachable_set, wc_reachable:
// traversal/level.rs:88-337 (LevelSearch), bfs.rs:34-111 and
// reachable.rs:18-90 on the device.
//
// A level is expanded by pushing (a warp per frontier node scans its row;
// each unvisited target is claimed with a compare-and-swap on its depth and
// every frontier node reaching it lowers its `via` with an atomic min) or by
// pulling (each unvisited node scans its reverse row, ascending, until it
// meets the frontier bitmap).  The reference's bfs always pushes, reporting
// for each node the first frontier node, in ascending order, whose row holds
// it: the smallest frontier predecessor.  Both forms here find exactly that
// node, so depths and `via` equal the reference's whichever form a level
// takes, and the visit order (by depth, then via, then node) follows from
// them.  reachable_set takes the reference's own switch (Beamer, α = 1,
// β = 24, level.rs:19-29, 184-211) so that its row order and its
// edges_traversed match too; bfs takes a GPU-tuned switch (pull when the
// frontier's rows outweigh a fourteenth of the unvisited nodes').
#include <algorithm>
#include <numeric>

#include "bfs.h"
#include "operand.h"
#include "semiring.cuh"

namespace wc {

__device__ inline bool bit_at(const uint32_t* b, uint32_t i) { return (b[i >> 5] >> (i & 31)) & 1; }

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
};

// The switch (level.rs:19-29, 184-211 for the reference's; a GPU-tuned one
// for bfs), evaluated where the level is planned.
struct SwitchArgs {
  uint32_t rule;  // SwitchRule
  uint32_t reverse_allowed;
  uint64_t n;
  uint64_t total_rdeg;
};

__host__ __device__ inline bool level_pulls(const SwitchArgs& a, uint64_t count, uint64_t mf,
                                            uint64_t visited_rdeg) {
  const uint64_t mu = a.total_rdeg - visited_rdeg;
  if (a.rule == REFERENCE_SWITCH) return a.reverse_allowed && count * 24 > a.n && mu < mf;
  return count * 24 > a.n && mf * 14 > mu;
}

struct Rows {  // the rows read in one direction: one CSR, or two for Both
  const uint32_t* off0;
  const uint32_t* tgt0;
  const uint32_t* off1;  // NULL unless Both
  const uint32_t* tgt1;
  __device__ uint32_t degree(uint32_t v) const {
    uint32_t d = __ldg(off0 + v + 1) - __ldg(off0 + v);
    if (off1) d += __ldg(off1 + v + 1) - __ldg(off1 + v);
    return d;
  }
};

// Appends v to the next frontier and marks it in the next frontier's
// bitmap: one atomic per warp for the lanes that admit a node this round.
__device__ inline void admit(uint32_t v, bool take, uint32_t* next, uint32_t* fnext,
                             LevelState* c, const Rows& adj, const Rows& radj) {
  const unsigned mask = __ballot_sync(0xffffffffu, take);
  if (!mask) return;
  const unsigned lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(&c->next_count, (uint32_t)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  unsigned long long d = 0, rd = 0;
  if (take) {
    next[base + __popc(mask & ((1u << lane) - 1))] = v;
    atomicOr(fnext + (v >> 5), 1u << (v & 31));
    d = adj.degree(v);
    rd = radj.degree(v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    d += __shfl_down_sync(0xffffffffu, d, o);
    rd += __shfl_down_sync(0xffffffffu, rd, o);
  }
  if (lane == 0) {
    atomicAdd(&c->next_deg, d);
    atomicAdd(&c->next_rdeg, rd);
  }
}

// What every kernel of a level is given.
struct LevelArgs {
  Rows adj, radj;
  LevelState* st;        // this level's state (st + 1: the next level's)
  const uint32_t* frontier;
  uint32_t* next;
  const uint32_t* fbits;  // this level's frontier as a bitmap
  uint32_t* fnext;        // the next level's bitmap (cleared)
  uint32_t* big;          // frontier rows too long for one warp
  uint32_t depth_next;
  uint32_t n;
  uint32_t* depth;
  unsigned long long* via;
  const uint64_t* filter;
};

// Levels queued per round trip to the host.
constexpr uint32_t kChunkLevels = 16;

// Rows longer than this are pushed by the whole grid (push_big_kernel):
// one warp per row would leave a hub's row to a single warp.
constexpr uint32_t kBigRow = 2048;

// One entry of a push: target v offered by frontier node u.
__device__ inline bool offer(const LevelArgs& a, uint32_t u, uint32_t v) {
  const bool allowed = !a.filter || ((a.filter[v >> 6] >> (v & 63)) & 1);
  if (!allowed) return false;
  const uint32_t d = a.depth[v];
  if (d != WC_UNREACHED && d != a.depth_next) return false;
  atomicMin(a.via + v, (unsigned long long)u);
  return d == WC_UNREACHED && atomicCAS(a.depth + v, WC_UNREACHED, a.depth_next) == WC_UNREACHED;
}

// Push: a warp per frontier node, lanes over its row entries; rows longer
// than kBigRow are listed for push_big_kernel instead.
__global__ void __launch_bounds__(256) push_kernel(LevelArgs a) {
  const LevelState& st = *a.st;
  if (st.count == 0 || st.pull) return;
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; f < st.count; f += warps) {
    const uint32_t u = a.frontier[f];
    if (a.adj.degree(u) > kBigRow) {
      if (lane == 0) a.big[atomicAdd(&a.st->big_count, 1u)] = u;
      continue;
    }
    for (int part = 0; part < 2; part++) {
      const uint32_t* off = part == 0 ? a.adj.off0 : a.adj.off1;
      const uint32_t* tgt = part == 0 ? a.adj.tgt0 : a.adj.tgt1;
      if (!off) break;
      const uint32_t lo = __ldg(off + u), hi = __ldg(off + u + 1);
      for (uint32_t e0 = lo; e0 < hi; e0 += 32) {
        const uint32_t e = e0 + lane;
        bool take = false;
        uint32_t v = 0;
        if (e < hi) {
          v = __ldg(tgt + e);
          take = offer(a, u, v);
        }
        admit(v, take, a.next, a.fnext, a.st, a.adj, a.radj);
      }
    }
  }
}

// Push of the long rows: each row's entries spread over every warp of the
// grid, the rows one after another.
__global__ void __launch_bounds__(256) push_big_kernel(LevelArgs a) {
  const LevelState& st = *a.st;
  if (st.count == 0 || st.pull || st.big_count == 0) return;
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t b = 0; b < st.big_count; b++) {
    const uint32_t u = a.big[b];
    for (int part = 0; part < 2; part++) {
      const uint32_t* off = part == 0 ? a.adj.off0 : a.adj.off1;
      const uint32_t* tgt = part == 0 ? a.adj.tgt0 : a.adj.tgt1;
      if (!off) break;
      const uint32_t lo = __ldg(off + u), hi = __ldg(off + u + 1);
      for (uint32_t e0 = lo + 32 * warp; e0 < hi; e0 += 32 * warps) {
        const uint32_t e = e0 + lane;
        bool take = false;
        uint32_t v = 0;
        if (e < hi) {
          v = __ldg(tgt + e);
          take = offer(a, u, v);
        }
        admit(v, take, a.next, a.fnext, a.st, a.adj, a.radj);
      }
    }
  }
}

// Pull: a thread per unvisited node, scanning its rows of `radj` (the
// opposite direction), in order, to the first frontier node.  For Both the
// smallest first hit of the two rows is `via` (what a push finds), while
// `edges` counts entries as the reference's pull scans them: the first row
// to its hit, or all of it and the second to its hit.
__global__ void __launch_bounds__(256) pull_kernel(LevelArgs a, int count_edges) {
  const LevelState& st = *a.st;
  if (st.count == 0 || !st.pull) return;
  unsigned long long scanned = 0;
  const uint32_t n = a.n;
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t rounds = (n + stride - 1) / stride;
  for (uint32_t r = 0; r < rounds; r++) {
    const uint32_t v = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
    bool take = false;
    if (v < n && a.depth[v] == WC_UNREACHED && (!a.filter || ((a.filter[v >> 6] >> (v & 63)) & 1))) {
      uint64_t best = WC_NO_VIA;
      bool counting = true;
      for (int part = 0; part < 2; part++) {
        const uint32_t* off = part == 0 ? a.radj.off0 : a.radj.off1;
        const uint32_t* tgt = part == 0 ? a.radj.tgt0 : a.radj.tgt1;
        if (!off) break;
        const uint32_t lo = __ldg(off + v), hi = __ldg(off + v + 1);
        for (uint32_t e = lo; e < hi; e++) {
          const uint32_t u = __ldg(tgt + e);
          if (counting) scanned++;
          if (bit_at(a.fbits, u)) {
            if (u < best) best = u;
            counting = false;
            break;
          }
        }
      }
      if (best != WC_NO_VIA) {
        a.depth[v] = a.depth_next;
        a.via[v] = best;
        take = true;
      }
    }
    admit(v, take, a.next, a.fnext, a.st, a.adj, a.radj);
  }
  if (count_edges) {
    for (int o = 16; o > 0; o >>= 1) scanned += __shfl_down_sync(0xffffffffu, scanned, o);
    if ((threadIdx.x & 31) == 0 && scanned) atomicAdd(&a.st->edges, scanned);
  }
}

// Closes a level: plans the next (its frontier, the switch's choice; an
// empty frontier past the depth cap or once the call is cancelled) and
// clears the bitmap the level after it will fill.
__global__ void level_end_kernel(LevelState* st, SwitchArgs sw, uint32_t next_is_last,
                                 uint32_t* fclear, uint32_t words, const int32_t* cancel) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x)
    fclear[i] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const LevelState& cur = st[0];
    LevelState& nx = st[1];
    const bool stop = cur.count == 0 || next_is_last || *(volatile const int32_t*)cancel;
    nx.count = stop ? 0u : cur.next_count;
    nx.mf = cur.next_deg;
    nx.visited_rdeg = cur.visited_rdeg + cur.next_rdeg;
    nx.pull = nx.count && level_pulls(sw, nx.count, nx.mf, nx.visited_rdeg);
  }
}

__global__ void set_bits_kernel(const uint32_t* nodes, uint32_t count, uint32_t* bits) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    atomicOr(bits + (nodes[i] >> 5), 1u << (nodes[i] & 31));
}

// For Both: whether node v sits in its via's forward row (a binary search;
// rows are ascending).  The reference scans the forward row, then the
// reverse row, so nodes of the forward row come first within a via.
__global__ void in_forward_row_kernel(uint32_t n, const uint32_t* depth,
                                      const unsigned long long* via, const uint32_t* off,
                                      const uint32_t* tgt, uint8_t* flag) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint8_t f = 1;
    if (depth[v] != WC_UNREACHED && depth[v] > 0 && via[v] != WC_NO_VIA) {
      uint32_t lo = off[via[v]], hi = off[via[v] + 1];
      while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        uint32_t t = tgt[mid];
        if (t == v) {
          f = 0;
          break;
        }
        if (t < v) lo = mid + 1;
        else hi = mid;
      }
    }
    flag[v] = f;
  }
}

__global__ void seed_kernel(const uint32_t* starts, uint32_t count, uint32_t* depth) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    depth[starts[i]] = 0;
}

static Rows rows_of(wc_version* v, int direction) {
  if (direction == WC_OUT)
    return Rows{v->fwd.offsets.as<uint32_t>(), v->fwd.targets.as<uint32_t>(), nullptr, nullptr};
  if (direction == WC_IN)
    return Rows{v->rev.offsets.as<uint32_t>(), v->rev.targets.as<uint32_t>(), nullptr, nullptr};
  return Rows{v->fwd.offsets.as<uint32_t>(), v->fwd.targets.as<uint32_t>(),
              v->rev.offsets.as<uint32_t>(), v->rev.targets.as<uint32_t>()};
}

static uint64_t host_degree(const wc_version* v, int direction, uint64_t node) {
  uint64_t d = 0;
  if (direction != WC_IN) d += v->host_offsets[node + 1] - v->host_offsets[node];
  if (direction != WC_OUT) d += v->host_rev_offsets[node + 1] - v->host_rev_offsets[node];
  return d;
}

wc_status Search::run(Ctx& ctx, int dir, const uint64_t* starts_in, uint64_t start_count,
                      uint32_t max_depth, const uint64_t* filter_host, SwitchRule rule) {
  wc_version* v = ctx.v;
  const uint64_t n = v->n;
  direction = dir;
  if (dir < WC_OUT || dir > WC_BOTH) return WC_INVALID_ARGUMENT;
  if (dir != WC_OUT && !v->reverse_given) return WC_REVERSE_CSR_MISSING;
  // The starts, repeats dropped, first occurrence kept (level.rs:125-147).
  std::vector<uint64_t> host_starts;
  if (start_count) {
    host_starts.resize(start_count);
    WC_CUDA(cudaMemcpy(host_starts.data(), starts_in, start_count * 8, cudaMemcpyDefault),
            ctx.detail);
  }
  for (uint64_t s : host_starts)
    if (s >= n) {
      if (ctx.detail) ctx.detail->node = s;
      return WC_NODE_OUTSIDE_ID_SPACE;
    }
  seeds.clear();
  {
    std::vector<uint64_t> sorted(host_starts);
    std::sort(sorted.begin(), sorted.end());
    std::vector<uint8_t> taken(sorted.size(), 0);
    for (uint64_t s : host_starts) {
      size_t at = std::lower_bound(sorted.begin(), sorted.end(), s) - sorted.begin();
      if (!taken[at]) {
        taken[at] = 1;
        seeds.push_back((uint32_t)s);
      }
    }
  }
  WC_TRY(ctx.scratch(POOL_BFS_DEPTH, n * 4, &depth));
  WC_TRY(ctx.scratch(POOL_BFS_VIA, n * 8, &via));
  WC_TRY(ctx.scratch(POOL_BFS_Q0, std::max<uint64_t>(n, 1) * 4, &queue[0]));
  WC_TRY(ctx.scratch(POOL_BFS_Q1, std::max<uint64_t>(n, 1) * 4, &queue[1]));
  const uint64_t words = (n + 31) / 32;
  WC_TRY(ctx.scratch(POOL_BFS_FBITS, std::max<uint64_t>(words, 1) * 4 * 2, &fbits));
  WC_TRY(ctx.scratch(POOL_BFS_COUNTERS, (kChunkLevels + 1) * sizeof(LevelState), &counters));
  WC_TRY(ctx.scratch(POOL_BFS_BIG, (v->m / kBigRow + 2) * 4 * (dir == WC_BOTH ? 2 : 1), &big));
  const uint64_t* filter_dev = nullptr;
  if (filter_host) {
    WC_TRY(ctx.scratch(POOL_BFS_FILTER, ((n + 63) / 64) * 8, &filter));
    WC_CUDA(cudaMemcpyAsync(filter->ptr, filter_host, ((n + 63) / 64) * 8, cudaMemcpyDefault,
                            ctx.stream), ctx.detail);
    filter_dev = filter->as<uint64_t>();
  }
  WC_CUDA(cudaMemsetAsync(depth->ptr, 0xff, n * 4, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(via->ptr, 0xff, n * 8, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(fbits->ptr, 0, std::max<uint64_t>(words, 1) * 4 * 2, ctx.stream),
          ctx.detail);
  const uint32_t count0 = (uint32_t)seeds.size();
  uint32_t* fb[2] = {fbits->as<uint32_t>(), fbits->as<uint32_t>() + std::max<uint64_t>(words, 1)};
  if (count0) {
    WC_CUDA(cudaMemcpyAsync(queue[0]->ptr, seeds.data(), count0 * 4, cudaMemcpyHostToDevice,
                            ctx.stream), ctx.detail);
    note_launch(), seed_kernel<<<(count0 + 255) / 256, 256, 0, ctx.stream>>>(queue[0]->as<uint32_t>(), count0,
                                                             depth->as<uint32_t>());
    note_launch(), set_bits_kernel<<<(count0 + 255) / 256, 256, 0, ctx.stream>>>(
        queue[0]->as<uint32_t>(), count0, fb[0]);
  }
  const Rows adj = rows_of(v, dir);
  const int rdir = dir == WC_OUT ? WC_IN : (dir == WC_IN ? WC_OUT : WC_BOTH);
  const Rows radj = rows_of(v, rdir);
  // Row lengths of the frontier (search direction) and of every node in
  // the opposite direction: what Beamer's switch compares.
  uint64_t mf = 0, visited_rdeg = 0;
  const uint64_t total_rdeg = (rdir == WC_BOTH ? 2 : 1) * v->m;
  for (uint32_t s : seeds) {
    mf += host_degree(v, dir, s);
    visited_rdeg += host_degree(v, rdir, s);
  }
  const SwitchArgs sw{(uint32_t)rule, (uint32_t)reverse_allowed, n, total_rdeg};
  stats = wc_traversal_stats{};
  stats.nodes_visited = count0;
  levels.clear();
  // The levels are queued kChunkLevels at a time with no round trip: each
  // level's kernels read its plan from the device (level_end_kernel writes
  // it), and those of a level with no frontier return at once.  The host
  // reads the chunk's plans back once, to go on or stop and for the stats.
  LevelState first{};
  first.count = max_depth > 0 ? count0 : 0;
  first.mf = mf;
  first.visited_rdeg = visited_rdeg;
  first.pull = first.count && level_pulls(sw, first.count, mf, visited_rdeg);
  LevelState* st = counters->as<LevelState>();
  const uint32_t blocks = max_blocks(8);
  const uint32_t pull_grid = std::max<uint32_t>(1, std::min<uint32_t>((uint32_t)((n + 255) / 256), blocks));
  const uint32_t end_grid = std::max<uint32_t>(1, std::min<uint32_t>((uint32_t)((words + 255) / 256), blocks));
  uint32_t d = 0;
  std::vector<LevelState> plan(kChunkLevels + 1);
  while (first.count > 0 && d < max_depth) {
    if (ctx.cancelled()) return WC_CANCELLED;
    WC_CUDA(cudaMemsetAsync(st, 0, (kChunkLevels + 1) * sizeof(LevelState), ctx.stream), ctx.detail);
    WC_CUDA(cudaMemcpyAsync(st, &first, sizeof first, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
    const uint32_t chunk = (uint32_t)std::min<uint64_t>(kChunkLevels, (uint64_t)max_depth - d);
    for (uint32_t q = 0; q < chunk; q++) {
      const uint32_t L = d + q;
      LevelArgs a{adj, radj, st + q, queue[L & 1]->as<uint32_t>(), queue[(L + 1) & 1]->as<uint32_t>(),
                  fb[L & 1], fb[(L + 1) & 1], big->as<uint32_t>(), L + 1, (uint32_t)n,
                  depth->as<uint32_t>(), via->as<unsigned long long>(), filter_dev};
      note_launch(), push_kernel<<<blocks, 256, 0, ctx.stream>>>(a);
      note_launch(), push_big_kernel<<<blocks, 256, 0, ctx.stream>>>(a);
      note_launch(), pull_kernel<<<pull_grid, 256, 0, ctx.stream>>>(a, 1);
      // The bitmap of level L + 2 is level L's: clear it for the admits of L + 1.
      note_launch(), level_end_kernel<<<end_grid, 256, 0, ctx.stream>>>(
          st + q, sw, L + 1 >= max_depth ? 1u : 0u, fb[L & 1], (uint32_t)words, v->cancel_dev);
    }
    WC_CUDA(cudaGetLastError(), ctx.detail);
    WC_CUDA(cudaMemcpyAsync(plan.data(), st, (chunk + 1) * sizeof(LevelState), cudaMemcpyDeviceToHost,
                            ctx.stream), ctx.detail);
    WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
    for (uint32_t q = 0; q < chunk; q++) {
      const LevelState& h = plan[q];
      if (h.count == 0) break;
      const bool pull = h.pull != 0;
      levels.push_back(Level{pull, h.count, h.mf, pull ? (uint64_t)h.edges : h.mf, h.next_count});
      stats.levels++;
      if (pull) stats.pulled_levels++;
      stats.edges_traversed += pull && rule == REFERENCE_SWITCH ? h.edges : h.mf;
      stats.nodes_visited += h.next_count;
      d++;
    }
    if (plan[chunk].count == 0) break;
    first = plan[chunk];
    first.next_deg = first.next_rdeg = first.edges = 0;
    first.next_count = first.big_count = 0;
  }
  return WC_OK;
}

// The visits in the reference's order: starts first (as given, repeats
// dropped), then level by level; a pushed level by (via, node), a pulled
// one (reachable_set only) by node.
wc_status Search::ordered(Ctx& ctx, std::vector<uint64_t>& rows, bool with_via) {
  const uint64_t n = ctx.v->n;
  std::vector<uint32_t> dh(n);
  std::vector<uint64_t> vh(n);
  WC_CUDA(cudaMemcpy(dh.data(), depth->ptr, n * 4, cudaMemcpyDeviceToHost), ctx.detail);
  WC_CUDA(cudaMemcpy(vh.data(), via->ptr, n * 8, cudaMemcpyDeviceToHost), ctx.detail);
  // Within a pushed level, nodes come by via, then by position in via's
  // rows: ascending for one CSR; for Both, the forward row's nodes first.
  std::vector<uint8_t> second_row(n, 0);
  if (direction == WC_BOTH && n) {
    DevBuf* flags;
    WC_TRY(ctx.scratch(POOL_BFS_FLAGS, n, &flags));
    note_launch(), in_forward_row_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(
        (uint32_t)n, depth->as<uint32_t>(), via->as<unsigned long long>(),
        ctx.v->fwd.offsets.as<uint32_t>(), ctx.v->fwd.targets.as<uint32_t>(), flags->as<uint8_t>());
    WC_CUDA(cudaMemcpyAsync(second_row.data(), flags->ptr, n, cudaMemcpyDeviceToHost, ctx.stream),
            ctx.detail);
    WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
  }
  std::vector<std::vector<std::pair<uint64_t, uint32_t>>> by_level(levels.size() + 1);
  for (uint64_t i = 0; i < n; i++)
    if (dh[i] != WC_UNREACHED && dh[i] > 0) {
      bool pulled = levels[dh[i] - 1].pulled && ordering_by_node_in_pulled;
      uint64_t key = pulled ? 0 : (vh[i] << 1) | second_row[i];
      by_level[dh[i]].push_back({key, (uint32_t)i});
    }
  rows.clear();
  auto put = [&](uint64_t node, uint32_t d, uint64_t via) {
    rows.push_back(node);
    if (with_via) {
      rows.push_back(d);
      rows.push_back(via);
    }
  };
  for (uint32_t s : seeds) put(s, 0, WC_NO_VIA);
  for (size_t d = 1; d < by_level.size(); d++) {
    auto& lv = by_level[d];
    std::sort(lv.begin(), lv.end());
    for (auto& p : lv) put(p.second, (uint32_t)d, vh[p.second]);
  }
  return WC_OK;
}

// The row entries a push-only search scans up to and including the entry
// that offers visit `index` of `rows` (the reference's order): every row of
// the levels before it, then in its level the rows of the frontier nodes
// before its `via`, and `via`'s rows up to the visit's node.
static wc_status scan_through(Ctx& ctx, const Search& s, const std::vector<uint64_t>& rows,
                              uint64_t index, uint64_t* edges_out) {
  wc_version* v = ctx.v;
  const int direction = s.direction;
  const uint64_t total = rows.size() / 3;
  const uint64_t node = rows[3 * index];
  const uint32_t d = (uint32_t)rows[3 * index + 1];
  uint64_t edges = 0;
  if (d > 0) {
    for (uint32_t l = 0; l + 1 < d; l++) edges += s.levels[l].frontier_entries;
    const uint64_t via = rows[3 * index + 2];
    std::vector<uint64_t> frontier;
    for (uint64_t r = 0; r < total; r++)
      if (rows[3 * r + 1] == d - 1) frontier.push_back(rows[3 * r]);
    std::sort(frontier.begin(), frontier.end());
    for (uint64_t f : frontier) {
      if (f == via) break;
      edges += host_degree(v, direction, f);
    }
    uint64_t pos = 0;
    bool found = false;
    for (int part = 0; part < 2 && !found; part++) {
      const bool use_fwd = part == 0 && direction != WC_IN;
      const bool use_rev = part == 0 ? direction == WC_IN : direction == WC_BOTH;
      if (!use_fwd && !use_rev) continue;
      const DevCsr& csr = use_fwd ? v->fwd : v->rev;
      const std::vector<uint64_t>& ho = use_fwd ? v->host_offsets : v->host_rev_offsets;
      const uint64_t lo = ho[via], hi = ho[via + 1];
      std::vector<uint32_t> row(hi - lo);
      if (hi > lo)
        WC_CUDA(cudaMemcpy(row.data(), csr.targets.as<uint32_t>() + lo, (hi - lo) * 4,
                           cudaMemcpyDeviceToHost), ctx.detail);
      for (uint64_t k = 0; k < row.size(); k++)
        if (row[k] == node) {
          pos += k + 1;
          found = true;
          break;
        }
      if (!found) pos += row.size();
    }
    edges += pos;
  }
  *edges_out = edges;
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_bfs(wc_version* v, const wc_call* call, wc_direction direction, const uint64_t* starts,
                 uint64_t start_count, const wc_limits* limits, const uint64_t* filter,
                 uint32_t* depth_out, uint64_t* via_out, wc_traversal_stats* stats) {
  if (!v || (start_count && !starts)) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  const uint32_t max_depth = limits ? limits->max_depth : WC_UNREACHED;
  const uint64_t max_results = limits ? limits->max_results : UINT64_MAX;
  if (max_results != UINT64_MAX) {
    // Truncation cuts the visit order: run the ordered form and scatter it.
    std::vector<uint64_t> rows(3 * (v->n + 1));
    uint64_t count = 0;
    WC_TRY(wc_bfs_visits(v, call, direction, starts, start_count, limits, filter, rows.data(),
                         v->n + 1, &count, stats));
    std::vector<uint32_t> d(v->n, WC_UNREACHED);
    std::vector<uint64_t> w(v->n, WC_NO_VIA);
    for (uint64_t r = 0; r < count; r++) {
      d[rows[3 * r]] = (uint32_t)rows[3 * r + 1];
      w[rows[3 * r]] = rows[3 * r + 2];
    }
    if (depth_out) WC_CUDA(cudaMemcpy(depth_out, d.data(), v->n * 4, cudaMemcpyDefault), ctx.detail);
    if (via_out) WC_CUDA(cudaMemcpy(via_out, w.data(), v->n * 8, cudaMemcpyDefault), ctx.detail);
    return WC_OK;
  }
  Search s;
  WC_TRY(s.run(ctx, direction, starts, start_count, max_depth, filter, GPU_SWITCH));
  WC_TRY(ctx.finish());
  if (depth_out)
    WC_CUDA(cudaMemcpyAsync(depth_out, s.depth->ptr, v->n * 4, cudaMemcpyDefault, ctx.stream),
            ctx.detail);
  if (via_out)
    WC_CUDA(cudaMemcpyAsync(via_out, s.via->ptr, v->n * 8, cudaMemcpyDefault, ctx.stream),
            ctx.detail);
  WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
  if (stats) *stats = s.stats;
  return WC_OK;
}

wc_status wc_bfs_visits(wc_version* v, const wc_call* call, wc_direction direction,
                        const uint64_t* starts, uint64_t start_count, const wc_limits* limits,
                        const uint64_t* filter, uint64_t* visits_out, uint64_t capacity,
                        uint64_t* count, wc_traversal_stats* stats) {
  if (!v || !count || (start_count && !starts)) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  const uint32_t max_depth = limits ? limits->max_depth : WC_UNREACHED;
  const uint64_t max_results = limits ? limits->max_results : UINT64_MAX;
  Search s;
  WC_TRY(s.run(ctx, direction, starts, start_count, max_depth, filter, GPU_SWITCH));
  WC_TRY(ctx.finish());
  std::vector<uint64_t> rows;
  WC_TRY(s.ordered(ctx, rows, true));
  uint64_t total = rows.size() / 3;
  wc_traversal_stats st = s.stats;
  if (max_results < total) {
    // bfs.rs:96-110: the visit past max_results is refused and the search
    // stops there.
    st.truncated = 1;
    st.nodes_visited = max_results;
    WC_TRY(scan_through(ctx, s, rows, max_results, &st.edges_traversed));
    total = max_results;
  }
  *count = total;
  if (visits_out) {
    uint64_t k = std::min(total, capacity);
    if (k) WC_CUDA(cudaMemcpy(visits_out, rows.data(), 3 * k * 8, cudaMemcpyDefault), ctx.detail);
  }
  if (stats) *stats = st;
  return WC_OK;
}

wc_status wc_reachable_set(wc_version* v, const wc_call* call, wc_direction direction,
                           const uint64_t* starts, uint64_t start_count, uint32_t max_depth,
                           uint64_t* nodes_out, uint64_t capacity, uint64_t* count,
                           wc_traversal_stats* stats) {
  if (!v || !count || (start_count && !starts)) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  Search s;
  s.reverse_allowed = v->reverse_given;
  s.ordering_by_node_in_pulled = true;
  WC_TRY(s.run(ctx, direction, starts, start_count, max_depth, nullptr, REFERENCE_SWITCH));
  WC_TRY(ctx.finish());
  std::vector<uint64_t> rows;
  WC_TRY(s.ordered(ctx, rows, false));
  *count = rows.size();
  uint64_t k = std::min<uint64_t>(rows.size(), capacity);
  if (nodes_out && k) WC_CUDA(cudaMemcpy(nodes_out, rows.data(), k * 8, cudaMemcpyDefault), ctx.detail);
  if (stats) *stats = s.stats;
  return WC_OK;
}

wc_status wc_reachable(wc_version* v, const wc_call* call, wc_direction direction, uint64_t start,
                       uint64_t target, uint32_t max_depth, int32_t* reached,
                       wc_traversal_stats* stats) {
  if (!v || !reached) return WC_INVALID_ARGUMENT;
  if (target >= v->n) {
    if (call && call->detail) call->detail->node = target;
    return WC_NODE_OUTSIDE_ID_SPACE;
  }
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  // reachable.rs:18-43: a push search from `start` that stops as soon as it
  // admits `target` (never pulled: it builds its edges without `pulling`).
  Search s;
  WC_TRY(s.run(ctx, direction, &start, 1, max_depth, nullptr, GPU_SWITCH));
  WC_TRY(ctx.finish());
  std::vector<uint64_t> rows;
  WC_TRY(s.ordered(ctx, rows, true));
  const uint64_t total = rows.size() / 3;
  wc_traversal_stats st = s.stats;
  *reached = 0;
  for (uint64_t r = 0; r < total; r++)
    if (rows[3 * r] == target) {
      *reached = 1;
      st.nodes_visited = r + 1;
      WC_TRY(scan_through(ctx, s, rows, r, &st.edges_traversed));
      break;
    }
  if (stats) *stats = st;
  return WC_OK;
}

}  // extern "C"
