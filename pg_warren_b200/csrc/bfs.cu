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
#include <string>

#include "bfs.h"
#include "operand.h"
#include "semiring.cuh"

namespace wc {

__device__ inline bool bit_at(const uint32_t* b, uint32_t i) { return (b[i >> 5] >> (i & 31)) & 1; }

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
  uint32_t* fclear;       // the previous level's bitmap, cleared here for the level after
  uint32_t fwords;
  uint32_t* big;          // frontier rows too long for one warp
  uint32_t big_cap;       // its entries: long rows from the front, huge ones from the back
  uint32_t depth_next;
  uint32_t n;
  uint32_t* depth;
  unsigned long long* via;
  const uint64_t* filter;
};

// Levels queued per round trip to the host.
constexpr uint32_t kChunkLevels = 16;

// Rows longer than this are pushed by a block each (push_big_kernel): one
// warp per row would leave a hub's row to a single warp.  Rows longer than
// kHugeRow are pushed by the whole grid, one after another.
constexpr uint32_t kBigRow = 2048;
constexpr uint32_t kHugeRow = 32768;

// The long-row list's entries: at most one per kBigRow entries of the rows
// read (both CSRs for Both).
inline uint32_t big_entries(uint64_t m, int dir) {
  return (uint32_t)((m / kBigRow + 2) * (dir == WC_BOTH ? 2 : 1));
}

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
__device__ inline void push_level(const LevelArgs& a) {
  const LevelState& st = *a.st;
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; f < st.count; f += warps) {
    const uint32_t u = a.frontier[f];
    const uint32_t deg = a.adj.degree(u);
    if (deg > kBigRow) {
      if (lane == 0) {
        if (deg > kHugeRow) a.big[a.big_cap - 1 - atomicAdd(&a.st->huge_count, 1u)] = u;
        else a.big[atomicAdd(&a.st->big_count, 1u)] = u;
      }
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

// Plans the level after st[0] in st[1]: its frontier (none past the depth
// cap or once the call is cancelled) and the switch's choice.
__device__ inline void plan_next(LevelState* st, const SwitchArgs& sw, uint32_t next_is_last,
                                 const int32_t* cancel) {
  const volatile LevelState& cur = st[0];
  LevelState& nx = st[1];
  const bool stop = cur.count == 0 || next_is_last || *(volatile const int32_t*)cancel;
  nx.count = stop ? 0u : cur.next_count;
  nx.mf = cur.next_deg;
  nx.visited_rdeg = cur.visited_rdeg + cur.next_rdeg;
  nx.pull = nx.count && level_pulls(sw, nx.count, nx.mf, nx.visited_rdeg);
}

// Push of the long rows: a huge row's entries spread over every warp of the
// grid, the huge rows one after another; then each long row over the warps
// of a team of blocks, the teams taking the long rows in turn.  Then the block
// that finishes last closes the level: it plans the next one.
__device__ inline void push_row_part(const LevelArgs& a, uint32_t u, uint32_t first_warp,
                                     uint32_t warp_stride) {
  const unsigned lane = threadIdx.x & 31;
  for (int part = 0; part < 2; part++) {
    const uint32_t* off = part == 0 ? a.adj.off0 : a.adj.off1;
    const uint32_t* tgt = part == 0 ? a.adj.tgt0 : a.adj.tgt1;
    if (!off) break;
    const uint32_t lo = __ldg(off + u), hi = __ldg(off + u + 1);
    for (uint32_t e0 = lo + 32 * first_warp; e0 < hi; e0 += 32 * warp_stride) {
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

__global__ void __launch_bounds__(256) push_big_kernel(LevelArgs a, SwitchArgs sw,
                                                       uint32_t next_is_last,
                                                       const int32_t* cancel) {
  const LevelState& st = *a.st;
  if (st.count == 0) return;  // no frontier: every later plan stays empty
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t huge = st.pull ? 0u : st.huge_count;
  for (uint32_t h = 0; h < huge; h++) push_row_part(a, a.big[a.big_cap - 1 - h], warp, warps);
  // Each long row gets a team of blocks: one when there are more rows than
  // blocks, else as many as share the grid evenly.
  const uint32_t big = st.pull ? 0u : st.big_count;
  if (big) {
    const uint32_t team = max(1u, gridDim.x / big);
    const uint32_t rows_at_once = gridDim.x / team;
    const uint32_t slot = blockIdx.x / team;
    const uint32_t wpb = blockDim.x >> 5;
    if (slot < rows_at_once)
      for (uint32_t b = slot; b < big; b += rows_at_once)
        push_row_part(a, a.big[b], (blockIdx.x % team) * wpb + (threadIdx.x >> 5), team * wpb);
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&a.st->done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    plan_next(a.st, sw, next_is_last, cancel);
  }
}

// Pull: a thread per unvisited node, scanning its rows of `radj` (the
// opposite direction), in order, to the first frontier node.  For Both the
// smallest first hit of the two rows is `via` (what a push finds), while
// `edges` counts entries as the reference's pull scans them: the first row
// to its hit, or all of it and the second to its hit.
__device__ inline void pull_level(const LevelArgs& a) {
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
  for (int o = 16; o > 0; o >>= 1) scanned += __shfl_down_sync(0xffffffffu, scanned, o);
  if ((threadIdx.x & 31) == 0 && scanned) atomicAdd(&a.st->edges, scanned);
}

// One launch a level: it pushes or pulls as the level's plan says (every
// block reads the same plan), and returns at once past the last frontier.
__global__ void __launch_bounds__(256) level_kernel(LevelArgs a) {
  const LevelState& st = *a.st;
  if (st.count == 0) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.fwords; i += gridDim.x * blockDim.x)
    a.fclear[i] = 0;
  if (st.pull) pull_level(a);
  else push_level(a);
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

// A search's state before its seeds: every depth unreached, every via
// none, both frontier bitmaps clear.
__global__ void bfs_fill_kernel(uint32_t* depth, unsigned long long* via, uint32_t n,
                                uint32_t* fbits, uint32_t fwords) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    depth[i] = WC_UNREACHED;
    via[i] = WC_NO_VIA;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < fwords; i += stride) fbits[i] = 0;
}

// The seeds (from the host's staging memory, read in place): depth 0, in
// the first queue and the first bitmap.
__global__ void bfs_seed_kernel(const uint32_t* seeds, uint32_t count, uint32_t* queue,
                                uint32_t* depth, uint32_t* fbits) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint32_t s = seeds[i];
    queue[i] = s;
    depth[s] = 0;
    atomicOr(fbits + (s >> 5), 1u << (s & 31));
  }
}

// A chunk's plans: the first from the host's staging memory, the rest zero.
__global__ void bfs_plan_kernel(const LevelState* first, LevelState* st, uint32_t count) {
  for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) st[i] = i == 0 ? *first : LevelState{};
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

wc_status Search::buffer(Ctx& ctx, int tag, uint64_t bytes, DevBuf** out) {
  if (!owned) return ctx.scratch(tag, bytes, out);
  DevBuf& b = (*owned)[tag];
  if (b.bytes < bytes) WC_TRY(b.alloc(ctx.budget, bytes, ctx.detail));
  *out = &b;
  return WC_OK;
}

wc_status Search::run(Ctx& ctx, int dir, const uint64_t* starts_in, uint64_t start_count,
                      uint32_t max_depth_in, const uint64_t* filter_host, SwitchRule rule) {
  WC_TRY(start(ctx, dir, starts_in, start_count, max_depth_in, filter_host, rule));
  return advance(ctx, UINT32_MAX);
}

wc_status Search::start(Ctx& ctx, int dir, const uint64_t* starts_in, uint64_t start_count,
                        uint32_t max_depth_in, const uint64_t* filter_host, SwitchRule rule) {
  wc_version* v = ctx.v;
  const uint64_t n = v->n;
  direction = dir;
  max_depth = max_depth_in;
  if (dir < WC_OUT || dir > WC_BOTH) return WC_INVALID_ARGUMENT;
  if (dir != WC_OUT && !v->reverse_given) return WC_REVERSE_CSR_MISSING;
  // The starts, repeats dropped, first occurrence kept (level.rs:125-147).
  std::vector<uint64_t> host_starts;
  if (start_count) {
    host_starts.resize(start_count);
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, starts_in) == cudaSuccess && pa.type == cudaMemoryTypeDevice) {
      WC_CUDA(cudaMemcpy(host_starts.data(), starts_in, start_count * 8, cudaMemcpyDeviceToHost),
              ctx.detail);
    } else {
      (void)cudaGetLastError();
      std::memcpy(host_starts.data(), starts_in, start_count * 8);
    }
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
  if (!depth_p) {
    WC_TRY(buffer(ctx, POOL_BFS_DEPTH, n * 4, &depth));
    depth_p = depth->as<uint32_t>();
  }
  if (!via_p) {
    WC_TRY(buffer(ctx, POOL_BFS_VIA, n * 8, &via));
    via_p = via->as<unsigned long long>();
  }
  WC_TRY(buffer(ctx, POOL_BFS_Q0, std::max<uint64_t>(n, 1) * 4, &queue[0]));
  WC_TRY(buffer(ctx, POOL_BFS_Q1, std::max<uint64_t>(n, 1) * 4, &queue[1]));
  const uint64_t words = (n + 31) / 32;
  WC_TRY(buffer(ctx, POOL_BFS_FBITS, std::max<uint64_t>(words, 1) * 4 * 3, &fbits));
  WC_TRY(buffer(ctx, POOL_BFS_COUNTERS, (kChunkLevels + 1) * sizeof(LevelState), &counters));
  WC_TRY(buffer(ctx, POOL_BFS_BIG, big_entries(v->m, dir) * 4, &big));
  filter = nullptr;
  if (filter_host) {
    WC_TRY(buffer(ctx, POOL_BFS_FILTER, ((n + 63) / 64) * 8, &filter));
    WC_CUDA(cudaMemcpyAsync(filter->ptr, filter_host, ((n + 63) / 64) * 8, cudaMemcpyDefault,
                            ctx.stream), ctx.detail);
  }
  // The device state (depths, vias, bitmaps, the seeds) is set up with the
  // first levels queued, in the same graph (enqueue_init).
  init_pending = true;
  const uint32_t count0 = (uint32_t)seeds.size();
  const int rdir = dir == WC_OUT ? WC_IN : (dir == WC_IN ? WC_OUT : WC_BOTH);
  // Row lengths of the frontier (search direction) and of every node in
  // the opposite direction: what Beamer's switch compares.
  uint64_t mf = 0, visited_rdeg = 0;
  const uint64_t total_rdeg = (rdir == WC_BOTH ? 2 : 1) * v->m;
  for (uint32_t s : seeds) {
    mf += host_degree(v, dir, s);
    visited_rdeg += host_degree(v, rdir, s);
  }
  sw = SwitchArgs{(uint32_t)rule, (uint32_t)reverse_allowed, n, total_rdeg};
  stats = wc_traversal_stats{};
  stats.nodes_visited = count0;
  levels.clear();
  depth_reached = 0;
  last_admitted = count0;
  next_plan = LevelState{};
  next_plan.count = max_depth > 0 ? count0 : 0;
  next_plan.mf = mf;
  next_plan.visited_rdeg = visited_rdeg;
  next_plan.pull = next_plan.count && level_pulls(sw, next_plan.count, mf, visited_rdeg);
  return WC_OK;
}

// Sets the device state up: every depth unreached, every via none, the
// bitmaps clear, the seeds at depth 0 in the first queue and bitmap.  The
// seeds come from the pinned staging area when they fit (so that the
// sequence can be captured and replayed), else from host memory.
wc_status Search::enqueue_init(Ctx& ctx, bool staged) {
  const uint64_t n = ctx.v->n;
  const uint64_t words = std::max<uint64_t>((n + 31) / 32, 1);
  const uint32_t count0 = (uint32_t)seeds.size();
  const uint64_t items = std::max<uint64_t>(n, 3 * words);
  const uint32_t fill_grid = (uint32_t)std::min<uint64_t>((items + 255) / 256, max_blocks(8));
  note_launch(), bfs_fill_kernel<<<fill_grid, 256, 0, ctx.stream>>>(
      depth_p, via_p, (uint32_t)n, fbits->as<uint32_t>(), (uint32_t)(3 * words));
  if (count0) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(ctx.v->stage_dev + kStagePayload);
    if (!staged) {
      WC_CUDA(cudaMemcpyAsync(queue[1]->ptr, seeds.data(), count0 * 4, cudaMemcpyHostToDevice,
                              ctx.stream), ctx.detail);
      src = queue[1]->as<uint32_t>();
    }
    note_launch(), bfs_seed_kernel<<<(count0 + 255) / 256, 256, 0, ctx.stream>>>(
        src, count0, queue[0]->as<uint32_t>(), depth_p, fbits->as<uint32_t>());
  }
  return cuda_status(cudaGetLastError(), ctx.detail, "bfs init");
}

wc_status Search::advance(Ctx& ctx, uint32_t max_levels, bool defer_last) {
  wc_version* v = ctx.v;
  const uint64_t n = v->n;
  const uint64_t words = (n + 31) / 32;
  const int dir = direction;
  const int rdir = dir == WC_OUT ? WC_IN : (dir == WC_IN ? WC_OUT : WC_BOTH);
  const Rows adj = rows_of(v, dir);
  const Rows radj = rows_of(v, rdir);
  // Three frontier bitmaps in turn: level L reads L % 3, fills (L + 1) % 3
  // and clears (L + 2) % 3, which the level before it read.
  const uint64_t fw = std::max<uint64_t>(words, 1);
  uint32_t* fb[3] = {fbits->as<uint32_t>(), fbits->as<uint32_t>() + fw,
                     fbits->as<uint32_t>() + 2 * fw};
  const uint64_t* filter_dev = filter ? filter->as<uint64_t>() : nullptr;
  LevelState* st = counters->as<LevelState>();
  const uint32_t blocks = max_blocks(8);
  // A push takes a warp per frontier node (rows longer than kBigRow go to
  // push_big_kernel), a pull a thread per node.
  const uint32_t big_cap = big_entries(v->m, dir);
  const uint32_t level_grid = std::max<uint32_t>(
      max_blocks(2), std::min<uint32_t>((uint32_t)((n + 255) / 256), blocks));
  uint32_t& d = depth_reached;
  const uint32_t stop_at = (uint32_t)std::min<uint64_t>(max_depth, (uint64_t)d + max_levels);
  static_assert((kChunkLevels + 1) * sizeof(LevelState) <= kStagePlanBytes, "plan staging");
  LevelState* plan = reinterpret_cast<LevelState*>(v->stage_host + kStagePlan);
  const bool seeds_fit = seeds.size() * 4 <= kStageBytes - kStagePayload;
  if (init_pending && (!seeds_fit || !(next_plan.count > 0 && d < stop_at))) {
    // No level follows, or the seeds do not fit the staging area: set the
    // state up on its own.
    init_pending = false;
    if (seeds_fit && !seeds.empty())
      std::memcpy(v->stage_host + kStagePayload, seeds.data(), seeds.size() * 4);
    WC_TRY(enqueue_init(ctx, seeds_fit));
  }
  // The levels are queued kChunkLevels at a time with no round trip: each
  // level's kernels read its plan from the device (push_big_kernel writes
  // it), and those of a level with no frontier return at once.  The host
  // reads the chunk's plans back once, to go on or stop and for the stats.
  while (next_plan.count > 0 && d < stop_at) {
    if (ctx.cancelled()) return WC_CANCELLED;
    const uint32_t chunk = std::min<uint32_t>(kChunkLevels, stop_at - d);
    const uint32_t d0 = d;
    const bool init = init_pending;
    init_pending = false;
    // What varies from call to call goes through the pinned staging area:
    // the first level's plan and the seeds.
    plan[0] = next_plan;
    if (init && !seeds.empty())
      std::memcpy(v->stage_host + kStagePayload, seeds.data(), seeds.size() * 4);
    // Every argument of the chunk's launches, so that a repeat of the same
    // shape replays the graph without capturing it.
    std::string args;
    auto put = [&](const void* p, size_t bytes) { args.append((const char*)p, bytes); };
    const uint64_t head[] = {chunk, d0, max_depth, init ? seeds.size() : UINT64_MAX, n,
                             (uint64_t)(uintptr_t)st, (uint64_t)(uintptr_t)v->cancel_dev,
                             (uint64_t)(uintptr_t)depth_p, (uint64_t)(uintptr_t)via_p,
                             (uint64_t)(uintptr_t)fbits->ptr, (uint64_t)(uintptr_t)queue[0]->ptr,
                             (uint64_t)(uintptr_t)queue[1]->ptr, (uint64_t)(uintptr_t)big->ptr,
                             (uint64_t)(uintptr_t)filter_dev, (uint64_t)(uintptr_t)adj.off0,
                             (uint64_t)(uintptr_t)adj.off1, (uint64_t)(uintptr_t)radj.off0,
                             (uint64_t)(uintptr_t)radj.off1, level_grid, blocks, big_cap,
                             (uint64_t)(uintptr_t)v->stage_host};
    put(head, sizeof head);
    put(&sw, sizeof sw);
    // The chunk's launches go out as one graph: a search of a few levels
    // costs one launch's latency, and a repeat of the same shape (the same
    // buffers, depth cap and seed count) no capture either.
    WC_TRY(ctx.run_cached("plainbfs/" + std::to_string(chunk), args, [&]() -> wc_status {
      if (init) WC_TRY(enqueue_init(ctx, true));
      note_launch(), bfs_plan_kernel<<<1, 32, 0, ctx.stream>>>(
          reinterpret_cast<const LevelState*>(v->stage_dev + kStagePlan), st, kChunkLevels + 1);
      for (uint32_t q = 0; q < chunk; q++) {
        const uint32_t L = d0 + q;
        LevelArgs a{adj, radj, st + q, queue[L & 1]->as<uint32_t>(),
                    queue[(L + 1) & 1]->as<uint32_t>(), fb[L % 3], fb[(L + 1) % 3],
                    fb[(L + 2) % 3], (uint32_t)fw, big->as<uint32_t>(), big_cap, L + 1, (uint32_t)n,
                    depth_p, via_p, filter_dev};
        note_launch(), level_kernel<<<level_grid, 256, 0, ctx.stream>>>(a);
        note_launch(), push_big_kernel<<<blocks, 256, 0, ctx.stream>>>(
            a, sw, L + 1 >= max_depth ? 1u : 0u, v->cancel_dev);
      }
      WC_CUDA(cudaMemcpyAsync(plan, st, (kChunkLevels + 1) * sizeof(LevelState),
                              cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
      return cuda_status(cudaGetLastError(), ctx.detail, "bfs levels");
    }));
    if (defer_last && d0 + chunk == stop_at) {
      // The last chunk there can be: the caller queues its own copies
      // behind it and waits once, then reads the plans (collect).
      pending_chunk = chunk;
      return WC_OK;
    }
    WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
    if (!absorb(plan, chunk)) break;
  }
  return WC_OK;
}

// Reads a chunk's plans back into the stats; whether the search goes on.
bool Search::absorb(const LevelState* plan, uint32_t chunk) {
  uint32_t& d = depth_reached;
  for (uint32_t q = 0; q < chunk; q++) {
    const LevelState& h = plan[q];
    if (h.count == 0) break;
    const bool pull = h.pull != 0;
    levels.push_back(Level{pull, h.count, h.mf, pull ? (uint64_t)h.edges : h.mf, h.next_count});
    stats.levels++;
    if (pull) stats.pulled_levels++;
    stats.edges_traversed += pull && sw.rule == REFERENCE_SWITCH ? h.edges : h.mf;
    stats.nodes_visited += h.next_count;
    last_admitted = h.next_count;
    d++;
  }
  const bool more = plan[chunk].count != 0;
  next_plan = plan[chunk];
  // A chunk cut short by max_levels leaves the next level planned; the
  // depth cap or an empty frontier leaves nothing to plan.
  if (d >= max_depth) next_plan.count = 0;
  next_plan.next_deg = next_plan.next_rdeg = next_plan.edges = 0;
  next_plan.next_count = next_plan.big_count = 0;
  return more;
}

void Search::collect(Ctx& ctx) {
  if (!pending_chunk) return;
  absorb(reinterpret_cast<const LevelState*>(ctx.v->stage_host + kStagePlan), pending_chunk);
  pending_chunk = 0;
}

// The visits in the reference's order: starts first (as given, repeats
// dropped), then level by level; a pushed level by (via, node), a pulled
// one (reachable_set only) by node.
wc_status Search::ordered(Ctx& ctx, std::vector<uint64_t>& rows, bool with_via) {
  const uint64_t n = ctx.v->n;
  std::vector<uint32_t> dh(n);
  std::vector<uint64_t> vh(n);
  WC_CUDA(cudaMemcpy(dh.data(), depth_p, n * 4, cudaMemcpyDeviceToHost), ctx.detail);
  WC_CUDA(cudaMemcpy(vh.data(), via_p, n * 8, cudaMemcpyDeviceToHost), ctx.detail);
  // Within a pushed level, nodes come by via, then by position in via's
  // rows: ascending for one CSR; for Both, the forward row's nodes first.
  std::vector<uint8_t> second_row(n, 0);
  if (direction == WC_BOTH && n) {
    DevBuf* flags;
    WC_TRY(ctx.scratch(POOL_BFS_FLAGS, n, &flags));
    note_launch(), in_forward_row_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(
        (uint32_t)n, depth_p, via_p,
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

// The row entries a pushed level scans up to and including the entry that
// offers `node` from `via`: the rows of the frontier nodes (ascending)
// before `via`, then `via`'s rows up to the node.
static wc_status push_scan(Ctx& ctx, int direction, const std::vector<uint64_t>& frontier_sorted,
                           uint64_t node, uint64_t via, uint64_t* edges_out) {
  wc_version* v = ctx.v;
  uint64_t edges = 0;
  for (uint64_t f : frontier_sorted) {
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
  *edges_out = edges + pos;
  return WC_OK;
}

// The row entries a push-only search scans up to and including the entry
// that offers visit `index` of `rows` (the reference's order): every row of
// the levels before it, then in its level the rows of the frontier nodes
// before its `via`, and `via`'s rows up to the visit's node.
static wc_status scan_through(Ctx& ctx, const Search& s, const std::vector<uint64_t>& rows,
                              uint64_t index, uint64_t* edges_out) {
  const uint64_t total = rows.size() / 3;
  const uint64_t node = rows[3 * index];
  const uint32_t d = (uint32_t)rows[3 * index + 1];
  uint64_t edges = 0;
  if (d > 0) {
    for (uint32_t l = 0; l + 1 < d; l++) edges += s.levels[l].frontier_entries;
    std::vector<uint64_t> frontier;
    for (uint64_t r = 0; r < total; r++)
      if (rows[3 * r + 1] == d - 1) frontier.push_back(rows[3 * r]);
    std::sort(frontier.begin(), frontier.end());
    uint64_t within = 0;
    WC_TRY(push_scan(ctx, s.direction, frontier, node, rows[3 * index + 2], &within));
    edges += within;
  }
  *edges_out = edges;
  return WC_OK;
}

// The rows of one level's admitted nodes, for ordering on the host:
// (node, via, 1 if the node is not in via's forward row (Both only)).
__global__ void level_rows_kernel(const uint32_t* nodes, uint32_t count,
                                  const unsigned long long* via, const uint32_t* off,
                                  const uint32_t* tgt, int both, unsigned long long* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint32_t v = nodes[i];
    const unsigned long long w = via[v];
    unsigned long long second = 0;
    if (both && w != WC_NO_VIA) {
      second = 1;
      uint32_t lo = off[w], hi = off[w + 1];
      while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        const uint32_t t = tgt[mid];
        if (t == v) {
          second = 0;
          break;
        }
        if (t < v) lo = mid + 1;
        else hi = mid;
      }
    }
    out[3 * (uint64_t)i] = v;
    out[3 * (uint64_t)i + 1] = w;
    out[3 * (uint64_t)i + 2] = second;
  }
}

// The row entries a pulled level (level.rs:243-282) scans through node
// `last`: each node not visited before the level (depth unreached, or the
// level's own `depth`), ascending, scans its opposite-direction rows in
// order up to its first frontier node (depth - 1), or all of them.
__global__ void pulled_scan_kernel(Rows radj, const uint32_t* depth, uint32_t level_depth,
                                   uint32_t last, unsigned long long* out) {
  unsigned long long sum = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= last; v += stride) {
    const uint32_t dv = depth[v];
    if (dv != WC_UNREACHED && dv != level_depth) continue;
    bool hit = false;
    for (int part = 0; part < 2 && !hit; part++) {
      const uint32_t* off = part == 0 ? radj.off0 : radj.off1;
      const uint32_t* tgt = part == 0 ? radj.tgt0 : radj.tgt1;
      if (!off) break;
      const uint32_t lo = __ldg(off + v), hi = __ldg(off + v + 1);
      for (uint32_t e = lo; e < hi; e++) {
        sum++;
        if (depth[__ldg(tgt + e)] == level_depth - 1) {
          hit = true;
          break;
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0 && sum) atomicAdd(out, sum);
}

}  // namespace wc

// traversal/bfs_cursor.rs:17-138 (BfsCursor): a search that lives across
// calls, one level per wc_bfs_cursor_next, with its own device buffers.
struct wc_bfs_cursor {
  wc_version* v = nullptr;
  wc::Search search;
  std::map<int, wc::DevBuf> bufs;  // the search's buffers, charged to the version's budget
  bool reachable = false;          // reachable_set's form: levels may be pulled
  uint64_t max_results = UINT64_MAX;
  uint64_t emitted = 0;            // visits handed out so far
  bool seeded = false, finished = false;
  std::vector<uint64_t> rows;      // the last level's visits: (node, depth, via)
  std::vector<uint64_t> frontier;  // the frontier it expanded, ascending
  bool pulled_order = false;       // the last level came in ascending node order
  wc_traversal_stats before{};     // the stats before the last level
  wc_traversal_stats stats{};
};

namespace wc {

// The stats of a search cut inside the cursor's last level: the visit at
// `index` of the level is the last one scanned (the refused one of a
// truncation, or the one a visitor broke at), `nodes` visits of the level
// were admitted.
static wc_status cut_stats(Ctx& ctx, wc_bfs_cursor* c, uint64_t index, uint64_t nodes,
                           bool truncated) {
  wc_traversal_stats st = c->stats;
  st.nodes_visited = c->before.nodes_visited + nodes;
  st.truncated = truncated ? 1 : 0;
  st.edges_traversed = c->before.edges_traversed;
  const uint64_t node = c->rows[3 * index];
  const uint32_t d = (uint32_t)c->rows[3 * index + 1];
  if (d > 0) {
    uint64_t within = 0;
    if (c->pulled_order) {
      const int dir = c->search.direction;
      const int rdir = dir == WC_OUT ? WC_IN : (dir == WC_IN ? WC_OUT : WC_BOTH);
      DevBuf* sum;
      WC_TRY(ctx.scratch(POOL_BFS_SCAN, 8, &sum));
      WC_CUDA(cudaMemsetAsync(sum->ptr, 0, 8, ctx.stream), ctx.detail);
      note_launch(), pulled_scan_kernel<<<max_blocks(8), 256, 0, ctx.stream>>>(
          rows_of(ctx.v, rdir), c->search.depth_p, d, (uint32_t)node,
          sum->as<unsigned long long>());
      WC_CUDA(cudaMemcpyAsync(&within, sum->ptr, 8, cudaMemcpyDeviceToHost, ctx.stream),
              ctx.detail);
      WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
    } else {
      WC_TRY(push_scan(ctx, c->search.direction, c->frontier, node, c->rows[3 * index + 2],
                       &within));
    }
    st.edges_traversed += within;
  }
  c->stats = st;
  return WC_OK;
}

// Expands the cursor's next level into c->rows, in the reference's order.
static wc_status cursor_level(Ctx& ctx, wc_bfs_cursor* c) {
  Search& s = c->search;
  c->pulled_order = false;
  if (!c->seeded) {
    c->seeded = true;
    c->rows.clear();
    c->frontier.clear();
    for (uint32_t x : s.seeds) c->rows.insert(c->rows.end(), {(uint64_t)x, 0, WC_NO_VIA});
    c->stats = s.stats;
    return WC_OK;
  }
  // The frontier this level expands: the last level's nodes, ascending.
  c->frontier.clear();
  for (size_t r = 0; r < c->rows.size(); r += 3) c->frontier.push_back(c->rows[r]);
  std::sort(c->frontier.begin(), c->frontier.end());
  c->rows.clear();
  const size_t had = s.levels.size();
  const uint32_t L = s.depth_reached;
  WC_TRY(s.advance(ctx, 1));
  WC_TRY(ctx.finish());
  c->stats = s.stats;
  if (s.levels.size() == had) return WC_OK;
  const Level& lv = s.levels.back();
  // bfs reports its levels as pushed whichever form ran; reachable_set
  // lists a pulled level by node.
  c->pulled_order = lv.pulled && c->reachable;
  const uint32_t k = lv.admitted;
  if (k == 0) return WC_OK;
  DevBuf* out;
  WC_TRY(ctx.scratch(POOL_BFS_ROWS, (uint64_t)k * 24, &out));
  const bool both = s.direction == WC_BOTH;
  note_launch(), level_rows_kernel<<<std::min<uint32_t>((k + 255) / 256, max_blocks(4)), 256, 0,
                                     ctx.stream>>>(
      s.queue[(L + 1) & 1]->as<uint32_t>(), k, s.via_p,
      ctx.v->fwd.offsets.as<uint32_t>(), ctx.v->fwd.targets.as<uint32_t>(), both ? 1 : 0,
      out->as<unsigned long long>());
  std::vector<uint64_t> raw((uint64_t)k * 3);
  WC_CUDA(cudaMemcpyAsync(raw.data(), out->ptr, (uint64_t)k * 24, cudaMemcpyDeviceToHost,
                          ctx.stream), ctx.detail);
  WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
  // A pushed level in the order reached: by via (frontier rows ascending),
  // then the forward row's nodes before the reverse row's (Both), then by
  // position in the row (rows are ascending); a pulled one by node.
  std::vector<uint32_t> idx(k);
  std::iota(idx.begin(), idx.end(), 0u);
  const bool by_node = c->pulled_order;
  std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
    const uint64_t* x = &raw[3 * (uint64_t)a];
    const uint64_t* y = &raw[3 * (uint64_t)b];
    if (!by_node) {
      if (x[1] != y[1]) return x[1] < y[1];
      if (x[2] != y[2]) return x[2] < y[2];
    }
    return x[0] < y[0];
  });
  c->rows.reserve((uint64_t)k * 3);
  for (uint32_t i : idx)
    c->rows.insert(c->rows.end(), {raw[3 * (uint64_t)i], (uint64_t)L + 1, raw[3 * (uint64_t)i + 1]});
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
  // Device outputs are searched in place (no copies out).
  const bool depth_dev = depth_out && is_device_pointer(depth_out);
  const bool via_dev = via_out && is_device_pointer(via_out);
  if (depth_dev) s.depth_p = depth_out;
  if (via_dev) s.via_p = reinterpret_cast<unsigned long long*>(via_out);
  WC_TRY(s.start(ctx, direction, starts, start_count, max_depth, filter, GPU_SWITCH));
  // The last chunk of levels, the copies out and the error word are waited
  // for once.
  WC_TRY(s.advance(ctx, UINT32_MAX, true));
  if (depth_out && !depth_dev)
    WC_CUDA(cudaMemcpyAsync(depth_out, s.depth_p, v->n * 4, cudaMemcpyDefault, ctx.stream),
            ctx.detail);
  if (via_out && !via_dev)
    WC_CUDA(cudaMemcpyAsync(via_out, s.via_p, v->n * 8, cudaMemcpyDefault, ctx.stream),
            ctx.detail);
  WC_TRY(ctx.finish());
  s.collect(ctx);
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

extern "C" {

wc_status wc_bfs_cursor_open(wc_version* v, const wc_call* call, wc_direction direction,
                             const uint64_t* starts, uint64_t start_count, const wc_limits* limits,
                             const uint64_t* filter, int32_t reachable_set, wc_bfs_cursor** out) {
  if (!v || !out || (start_count && !starts)) return WC_INVALID_ARGUMENT;
  *out = nullptr;
  const uint32_t max_depth = limits ? limits->max_depth : WC_UNREACHED;
  const uint64_t max_results = limits ? limits->max_results : UINT64_MAX;
  // reachable_set takes no filter and no result limit (reachable.rs:48-58).
  if (reachable_set && (filter || max_results != UINT64_MAX)) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  std::unique_ptr<wc_bfs_cursor> c(new wc_bfs_cursor);
  c->v = v;
  c->reachable = reachable_set != 0;
  c->max_results = max_results;
  c->search.owned = &c->bufs;
  if (c->reachable) {
    c->search.reverse_allowed = v->reverse_given;
    c->search.ordering_by_node_in_pulled = true;
  }
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  WC_TRY(c->search.start(ctx, direction, starts, start_count, max_depth, filter,
                         c->reachable ? REFERENCE_SWITCH : GPU_SWITCH));
  WC_TRY(ctx.finish());
  v->cursors.fetch_add(1);
  *out = c.release();
  return WC_OK;
}

wc_status wc_bfs_cursor_next(wc_bfs_cursor* c, const wc_call* call, uint64_t* count,
                             int32_t* more) {
  if (!c || !count) return WC_INVALID_ARGUMENT;
  *count = 0;
  if (more) *more = 0;
  if (c->finished) {
    c->rows.clear();
    return WC_OK;
  }
  wc_version* v = c->v;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  // A level that fails (cancelled, timed out, out of memory) ends the
  // cursor: its device state is no longer one the search can go on from.
  auto fail = [&](wc_status st) {
    c->finished = true;
    c->rows.clear();
    return st;
  };
  // Interrupts are polled before any work (interrupts.rs; the seed's first
  // admission polls, and so does each expansion).
  if (ctx.cancelled()) return fail(WC_CANCELLED);
  if (const wc_status st = ctx.begin(); st != WC_OK) return fail(st);
  c->before = c->stats;
  if (const wc_status st = cursor_level(ctx, c); st != WC_OK) return fail(st);
  const uint64_t k = c->rows.size() / 3;
  if (c->max_results - c->emitted < k) {
    // bfs.rs:96-110: the visit past max_results is refused and the search
    // stops there.
    const uint64_t keep = c->max_results - c->emitted;
    WC_TRY(cut_stats(ctx, c, keep, keep, true));
    c->rows.resize(3 * keep);
    c->finished = true;
  } else {
    c->finished = c->search.exhausted();
  }
  c->emitted += c->rows.size() / 3;
  *count = c->rows.size() / 3;
  if (more) *more = c->finished ? 0 : 1;
  return WC_OK;
}

wc_status wc_bfs_cursor_read(const wc_bfs_cursor* c, uint64_t first, uint64_t rows,
                             uint64_t* visits_out) {
  if (!c || (rows && !visits_out)) return WC_INVALID_ARGUMENT;
  const uint64_t have = c->rows.size() / 3;
  if (first > have || rows > have - first) return WC_INVALID_ARGUMENT;
  if (rows)
    WC_CUDA(cudaMemcpy(visits_out, c->rows.data() + 3 * first, rows * 24, cudaMemcpyDefault),
            nullptr);
  return WC_OK;
}

wc_status wc_bfs_cursor_stop(wc_bfs_cursor* c, const wc_call* call, uint64_t consumed) {
  if (!c) return WC_INVALID_ARGUMENT;
  const uint64_t have = c->rows.size() / 3;
  if (consumed == 0 || consumed > have) return WC_INVALID_ARGUMENT;
  wc_version* v = c->v;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  // A visitor that breaks admits the visit it broke at (Admission::
  // AdmitAndStop, level.rs:304-324): the search stops there, not truncated.
  WC_TRY(cut_stats(ctx, c, consumed - 1, consumed, false));
  c->rows.resize(3 * consumed);
  c->emitted = c->emitted - have + consumed;
  c->finished = true;
  return WC_OK;
}

wc_status wc_bfs_cursor_stats(const wc_bfs_cursor* c, wc_traversal_stats* stats) {
  if (!c || !stats) return WC_INVALID_ARGUMENT;
  *stats = c->stats;
  return WC_OK;
}

void wc_bfs_cursor_destroy(wc_bfs_cursor* c) {
  if (!c) return;
  wc_version* v = c->v;
  {
    std::lock_guard<std::recursive_mutex> lock(v->mu);
    cudaSetDevice(v->device);
    if (v->stream) cudaStreamSynchronize(v->stream);
    c->bufs.clear();
  }
  v->cursors.fetch_sub(1);
  delete c;
}

}  // extern "C"
