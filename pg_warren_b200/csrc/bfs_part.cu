// bfs_part.cu — one rank's part of a row-partitioned level search (no
// reference counterpart: warren-core searches on one host).  The search of
// traversal/level.rs:100-200 (LevelSearch) with its rows cut into one range
// per rank; every rank holds the whole version and the whole frontier, and
// owns the visited bits and depths of its rows.  A level:
//
//   - each rank finds the rows of its range that the level reaches — pulled
//     (its unvisited rows scan their in-entries for a frontier node) or
//     pushed (the whole frontier's rows scanned for entries into its range),
//     the same choice on every rank from the frontier's summed out-edges;
//   - the rank settles them (visited, depth = level + 1) and reports how many
//     and their out-edges;
//   - between levels the caller sums those two counts over the ranks and
//     gathers the parts' words of the next frontier bitmap (n/8 bytes).
//
// The depths are a level search's, so every node's depth equals wc_bfs's
// (the set of nodes at each depth does not depend on push or pull).
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "operand.h"
#include "runtime.cuh"

namespace wc {

namespace {

// The pull and push adjacency of a search in `dir`: pulling a row reads the
// entries that reach it, pushing a frontier row reads those leaving it.
struct Adj {
  const uint32_t* off[2];
  const uint32_t* tgt[2];
  int count;  // 1, or 2 for WC_BOTH
};

Adj pull_adj(const wc_version* v, int dir) {
  Adj a{};
  if (dir == WC_OUT) a = Adj{{v->rev.offsets.as<uint32_t>()}, {v->rev.targets.as<uint32_t>()}, 1};
  else if (dir == WC_IN) a = Adj{{v->fwd.offsets.as<uint32_t>()}, {v->fwd.targets.as<uint32_t>()}, 1};
  else
    a = Adj{{v->rev.offsets.as<uint32_t>(), v->fwd.offsets.as<uint32_t>()},
            {v->rev.targets.as<uint32_t>(), v->fwd.targets.as<uint32_t>()}, 2};
  return a;
}

Adj push_adj(const wc_version* v, int dir) {
  Adj a{};
  if (dir == WC_OUT) a = Adj{{v->fwd.offsets.as<uint32_t>()}, {v->fwd.targets.as<uint32_t>()}, 1};
  else if (dir == WC_IN) a = Adj{{v->rev.offsets.as<uint32_t>()}, {v->rev.targets.as<uint32_t>()}, 1};
  else
    a = Adj{{v->fwd.offsets.as<uint32_t>(), v->rev.offsets.as<uint32_t>()},
            {v->fwd.targets.as<uint32_t>(), v->rev.targets.as<uint32_t>()}, 2};
  return a;
}

__device__ inline bool bit_of(const uint32_t* bits, uint32_t i) {
  return (__ldg(bits + (i >> 5)) >> (i & 31)) & 1u;
}

// Sets the starts' frontier bits (every start: the frontier is global) and
// the visited bits and depth 0 of the starts in [lo, hi).
__global__ void bpart_seed_kernel(const uint64_t* starts, uint64_t count, uint32_t lo,
                                  uint32_t hi, uint32_t* F, uint32_t* visited, uint32_t* depth) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = (uint32_t)starts[i];
    atomicOr(F + (s >> 5), 1u << (s & 31));
    if (s >= lo && s < hi) {
      atomicOr(visited + (s >> 5), 1u << (s & 31));
      depth[s] = 0;
    }
  }
}

// The nodes and push-side out-edges of the bitmap's words [w0, w1):
// sums[0] += nodes, sums[1] += edges.
__global__ void __launch_bounds__(256) bpart_count_kernel(const uint32_t* F, uint32_t w0,
                                                          uint32_t w1, Adj push,
                                                          unsigned long long* sums) {
  unsigned long long nodes = 0, edges = 0;
  for (uint32_t w = w0 + blockIdx.x * blockDim.x + threadIdx.x; w < w1;
       w += gridDim.x * blockDim.x) {
    uint32_t b = F[w];
    nodes += __popc(b);
    while (b) {
      const uint32_t u = w * 32 + __ffs(b) - 1;
      b &= b - 1;
      for (int k = 0; k < push.count; k++) edges += __ldg(push.off[k] + u + 1) - __ldg(push.off[k] + u);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    nodes += __shfl_down_sync(0xffffffffu, nodes, o);
    edges += __shfl_down_sync(0xffffffffu, edges, o);
  }
  if ((threadIdx.x & 31) == 0 && (nodes || edges)) {
    atomicAdd(sums, nodes);
    atomicAdd(sums + 1, edges);
  }
}

// Pull: warp g of the grid takes the 32 rows of word w0 + g; each unvisited
// row of [lo, hi) looks for an entry from a frontier node.  A row of at most
// 32 entries (per adjacency) is scanned by its own lane; longer rows by the
// whole warp, 32 entries a step, stopping at the first hit.
__global__ void __launch_bounds__(256) bpart_pull_kernel(Adj pull, const uint32_t* F,
                                                         const uint32_t* visited, uint32_t lo,
                                                         uint32_t hi, uint32_t* N) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t w_lo = lo >> 5, w_hi = (hi + 31) >> 5;
  for (uint32_t w = w_lo + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < w_hi; w += warps) {
    const uint32_t r = w * 32 + lane;
    const bool cand = r >= lo && r < hi && !((visited[w] >> lane) & 1u);
    bool found = false, longrow = false;
    if (cand) {
      for (int k = 0; k < pull.count && !found; k++) {
        const uint32_t e0 = __ldg(pull.off[k] + r), e1 = __ldg(pull.off[k] + r + 1);
        if (e1 - e0 > 32) {
          longrow = true;
          continue;
        }
        for (uint32_t e = e0; e < e1; e++)
          if (bit_of(F, __ldg(pull.tgt[k] + e))) {
            found = true;
            break;
          }
      }
    }
    uint32_t longs = __ballot_sync(0xffffffffu, longrow && !found);
    while (longs) {
      const unsigned src = __ffs(longs) - 1;
      longs &= longs - 1;
      const uint32_t row = w * 32 + src;
      bool hit = false;
      for (int k = 0; k < pull.count && !hit; k++) {
        const uint32_t e0 = __ldg(pull.off[k] + row), e1 = __ldg(pull.off[k] + row + 1);
        if (e1 - e0 <= 32) continue;  // scanned by its lane
        for (uint32_t e = e0; e < e1 && !hit; e += 32) {
          const bool h = e + lane < e1 && bit_of(F, __ldg(pull.tgt[k] + e + lane));
          hit = __ballot_sync(0xffffffffu, h) != 0;
        }
      }
      if (hit && lane == src) found = true;
    }
    const uint32_t word = __ballot_sync(0xffffffffu, found);
    if (lane == 0) N[w] = word;
  }
}

// Push: warp g takes frontier word g (of every part: the frontier is
// global); for each frontier node its lanes stride over the node's entries
// and set the bits of unvisited targets in [lo, hi).
__global__ void __launch_bounds__(256) bpart_push_kernel(Adj push, const uint32_t* F,
                                                         uint32_t words, const uint32_t* visited,
                                                         uint32_t lo, uint32_t hi, uint32_t* N) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < words; w += warps) {
    uint32_t b = __ldg(F + w);
    while (b) {
      const uint32_t u = w * 32 + __ffs(b) - 1;
      b &= b - 1;
      for (int k = 0; k < push.count; k++) {
        const uint32_t e0 = __ldg(push.off[k] + u), e1 = __ldg(push.off[k] + u + 1);
        for (uint32_t e = e0 + lane; e < e1; e += 32) {
          const uint32_t t = __ldg(push.tgt[k] + e);
          if (t >= lo && t < hi && !((visited[t >> 5] >> (t & 31)) & 1u))
            atomicOr(N + (t >> 5), 1u << (t & 31));
        }
      }
    }
  }
}

// The level's rows of [lo, hi) are settled: visited, depth = level + 1, and
// their count and push-side out-edges summed into sums[0], sums[1].
__global__ void __launch_bounds__(256) bpart_settle_kernel(uint32_t* N, uint32_t* visited,
                                                           uint32_t* depth, uint32_t lo,
                                                           uint32_t hi, uint32_t next_depth,
                                                           Adj push, unsigned long long* sums) {
  unsigned long long nodes = 0, edges = 0;
  const uint32_t w_lo = lo >> 5, w_hi = (hi + 31) >> 5;
  for (uint32_t w = w_lo + blockIdx.x * blockDim.x + threadIdx.x; w < w_hi;
       w += gridDim.x * blockDim.x) {
    uint32_t b = N[w] & ~visited[w];
    N[w] = b;
    if (!b) continue;
    visited[w] |= b;
    nodes += __popc(b);
    while (b) {
      const uint32_t u = w * 32 + __ffs(b) - 1;
      b &= b - 1;
      depth[u] = next_depth;
      for (int k = 0; k < push.count; k++) edges += __ldg(push.off[k] + u + 1) - __ldg(push.off[k] + u);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    nodes += __shfl_down_sync(0xffffffffu, nodes, o);
    edges += __shfl_down_sync(0xffffffffu, edges, o);
  }
  if ((threadIdx.x & 31) == 0 && (nodes || edges)) {
    atomicAdd(sums, nodes);
    atomicAdd(sums + 1, edges);
  }
}

__global__ void bpart_fill_kernel(uint32_t* p, uint32_t lo, uint32_t hi, uint32_t value) {
  for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    p[i] = value;
}

// A level pushes while the frontier's out-edges are below the scanned
// entries over this divisor; every rank decides from the same sums.
constexpr uint64_t kPartPushDivisor = 32;

uint32_t grid_for(uint64_t items, uint32_t per_block) {
  const uint64_t g = (items + per_block - 1) / per_block;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(g, max_blocks(8)));
}

}  // namespace

// The parts' first rows for a search in `dir`: each part takes about an
// equal share of the rows' pull entries plus one per row, cut at multiples
// of 64 rows so that every 64-bit word of a bitmap has one owner.  Kept per
// (version, direction, parts): the offsets are read back only the first
// time.
static std::map<std::tuple<const wc_version*, int, uint32_t>, std::vector<uint64_t>> g_cuts;
static std::mutex g_cuts_mu;

static wc_status compute_bfs_part_cuts(wc_version* v, int dir, uint32_t parts,
                                       std::vector<uint64_t>& cut, wc_error_detail* detail);

static wc_status bfs_part_cuts(wc_version* v, int dir, uint32_t parts, std::vector<uint64_t>& cut,
                               wc_error_detail* detail) {
  const auto key = std::make_tuple((const wc_version*)v, dir, parts);
  {
    std::lock_guard<std::mutex> lock(g_cuts_mu);
    auto it = g_cuts.find(key);
    if (it != g_cuts.end()) {
      cut = it->second;
      return WC_OK;
    }
  }
  WC_TRY(compute_bfs_part_cuts(v, dir, parts, cut, detail));
  std::lock_guard<std::mutex> lock(g_cuts_mu);
  g_cuts[key] = cut;
  return WC_OK;
}

static wc_status compute_bfs_part_cuts(wc_version* v, int dir, uint32_t parts,
                                       std::vector<uint64_t>& cut, wc_error_detail* detail) {
  const uint64_t n = v->n;
  std::vector<uint64_t> work(n + 1, 0);
  std::vector<uint32_t> off(n + 1);
  const DevCsr* csrs[2] = {dir == WC_IN ? &v->fwd : &v->rev, dir == WC_BOTH ? &v->fwd : nullptr};
  for (const DevCsr* c : csrs) {
    if (!c) continue;
    WC_CUDA(cudaMemcpy(off.data(), c->offsets.ptr, (n + 1) * 4, cudaMemcpyDeviceToHost), detail);
    for (uint64_t i = 0; i <= n; i++) work[i] += off[i];
  }
  for (uint64_t i = 0; i <= n; i++) work[i] += i;
  cut.assign(parts + 1, n);
  cut[0] = 0;
  const uint64_t total = work[n];
  for (uint32_t p = 1; p < parts; p++) {
    const uint64_t goal = (total * p + parts - 1) / parts;
    uint64_t r = std::lower_bound(work.begin(), work.end(), goal) - work.begin();
    r = std::min<uint64_t>((r + 63) / 64 * 64, n);
    cut[p] = std::max(r, cut[p - 1]);
  }
  return WC_OK;
}

namespace {

struct PartSearch {
  int dir = WC_OUT;
  uint32_t lo = 0, hi = 0;
  uint32_t max_depth = 0;
  uint64_t* frontier2 = nullptr;  // the caller's: 2 × words
  uint64_t words = 0;
  DevBuf *visited = nullptr, *depth = nullptr, *sums = nullptr;  // the version's pool
};

std::map<const wc_version*, std::unique_ptr<PartSearch>> g_searches;
std::mutex g_searches_mu;

PartSearch* search_of(const wc_version* v) {
  std::lock_guard<std::mutex> lock(g_searches_mu);
  auto it = g_searches.find(v);
  return it == g_searches.end() ? nullptr : it->second.get();
}

uint32_t* frontier_half(PartSearch* ps, uint32_t level) {
  return reinterpret_cast<uint32_t*>(ps->frontier2 + (level & 1) * ps->words);
}

}  // namespace

void bfs_part_forget(const wc_version* v) {
  {
    std::lock_guard<std::mutex> lock(g_searches_mu);
    g_searches.erase(v);
  }
  std::lock_guard<std::mutex> lock(g_cuts_mu);
  for (auto it = g_cuts.begin(); it != g_cuts.end();)
    it = std::get<0>(it->first) == v ? g_cuts.erase(it) : std::next(it);
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_bfs_part_rows(wc_version* v, wc_direction direction, uint32_t parts,
                           uint64_t* row_bounds) {
  if (!v || parts == 0 || !row_bounds || direction < WC_OUT || direction > WC_BOTH)
    return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), nullptr);
  std::vector<uint64_t> cut;
  WC_TRY(bfs_part_cuts(v, direction, parts, cut, nullptr));
  std::copy(cut.begin(), cut.end(), row_bounds);
  return WC_OK;
}

wc_status wc_bfs_part_begin(wc_version* v, const wc_call* call, wc_direction direction,
                            const uint64_t* starts, uint64_t start_count, uint32_t max_depth,
                            uint32_t parts, uint32_t part, uint64_t* frontier2,
                            wc_bfs_part_info* info) {
  if (!v || !frontier2 || !info || (start_count && !starts) || parts == 0 || part >= parts ||
      direction < WC_OUT || direction > WC_BOTH)
    return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  if (!is_device_pointer(frontier2)) {
    set_message(ctx.detail, "the frontier bitmaps must be device memory");
    return WC_INVALID_ARGUMENT;
  }
  const uint64_t n = v->n;
  // The starts are checked before anything runs (NodeOutsideIdSpace).
  std::vector<uint64_t> host(start_count);
  if (start_count)
    WC_CUDA(cudaMemcpy(host.data(), starts, start_count * 8, cudaMemcpyDefault), ctx.detail);
  for (uint64_t s : host)
    if (s >= n) {
      if (ctx.detail) ctx.detail->node = s;
      set_message(ctx.detail, "start %llu is outside the id space of %llu nodes",
                  (unsigned long long)s, (unsigned long long)n);
      return WC_NODE_OUTSIDE_ID_SPACE;
    }
  std::vector<uint64_t> cut;
  WC_TRY(bfs_part_cuts(v, direction, parts, cut, ctx.detail));
  auto ps = std::make_unique<PartSearch>();
  ps->dir = direction;
  ps->lo = (uint32_t)cut[part];
  ps->hi = (uint32_t)cut[part + 1];
  ps->max_depth = max_depth;
  ps->frontier2 = frontier2;
  ps->words = (n + 63) / 64;
  const uint64_t words32 = 2 * ps->words;
  // Pooled with the version (kept between searches), so a search allocates
  // only when it needs more than the last one did.
  WC_TRY(ctx.scratch(POOL_PART_VISITED, std::max<uint64_t>(words32, 1) * 4, &ps->visited));
  WC_TRY(ctx.scratch(POOL_PART_DEPTH, std::max<uint64_t>(n, 1) * 4, &ps->depth));
  WC_TRY(ctx.scratch(POOL_PART_SUMS, 64, &ps->sums));
  DevBuf* starts_dev = nullptr;
  if (start_count) WC_TRY(ctx.scratch(POOL_PART_STARTS, start_count * 8, &starts_dev));
  WC_TRY(ctx.begin());
  if (start_count)
    WC_CUDA(cudaMemcpyAsync(starts_dev->ptr, host.data(), start_count * 8, cudaMemcpyHostToDevice,
                            ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(frontier2, 0, 2 * ps->words * 8, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(ps->visited->ptr, 0, std::max<uint64_t>(words32, 1) * 4, ctx.stream),
          ctx.detail);
  WC_CUDA(cudaMemsetAsync(ps->sums->ptr, 0, 64, ctx.stream), ctx.detail);
  if (ps->hi > ps->lo)
    note_launch(), bpart_fill_kernel<<<grid_for(ps->hi - ps->lo, 256), 256, 0, ctx.stream>>>(
        ps->depth->as<uint32_t>(), ps->lo, ps->hi, WC_UNREACHED);
  uint32_t* F = frontier_half(ps.get(), 0);
  if (start_count)
    note_launch(), bpart_seed_kernel<<<grid_for(start_count, 256), 256, 0, ctx.stream>>>(
        starts_dev->as<uint64_t>(), start_count, ps->lo, ps->hi, F, ps->visited->as<uint32_t>(),
        ps->depth->as<uint32_t>());
  // Level 0's frontier, counted over the whole bitmap (the same on every part).
  note_launch(), bpart_count_kernel<<<grid_for(words32, 256), 256, 0, ctx.stream>>>(
      F, 0, (uint32_t)words32, push_adj(v, direction), ps->sums->as<unsigned long long>());
  WC_CUDA(cudaGetLastError(), ctx.detail);
  WC_TRY(ctx.finish());
  unsigned long long sums[2];
  WC_CUDA(cudaMemcpy(sums, ps->sums->ptr, 16, cudaMemcpyDeviceToHost), ctx.detail);
  info->row_begin = ps->lo;
  info->row_end = ps->hi;
  info->id_space = n;
  info->words = ps->words;
  info->frontier = sums[0];
  info->frontier_edges = sums[1];
  std::lock_guard<std::mutex> slock(g_searches_mu);
  g_searches[v] = std::move(ps);
  return WC_OK;
}

wc_status wc_bfs_part_step(wc_version* v, const wc_call* call, uint32_t level,
                           uint64_t frontier_edges, uint64_t* sums) {
  if (!v || !sums) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  PartSearch* ps = search_of(v);
  if (!ps) return WC_INVALID_ARGUMENT;
  if (level >= ps->max_depth) {
    set_message(call ? call->detail : nullptr, "level %u is at the depth limit %u", level,
                ps->max_depth);
    return WC_INVALID_ARGUMENT;
  }
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  const uint32_t* F = frontier_half(ps, level);
  uint32_t* N = frontier_half(ps, level + 1);
  unsigned long long* acc = ps->sums->as<unsigned long long>();
  WC_CUDA(cudaMemsetAsync(acc, 0, 16, ctx.stream), ctx.detail);
  if (ps->hi > ps->lo) {
    const uint32_t w_lo = ps->lo / 32, w_hi = (ps->hi + 31) / 32;
    const uint64_t scanned = (ps->dir == WC_BOTH ? 2 : 1) * v->m;
    const bool push = frontier_edges * kPartPushDivisor < scanned;
    uint32_t* visited = ps->visited->as<uint32_t>();
    if (push) {
      WC_CUDA(cudaMemsetAsync(N + w_lo, 0, (uint64_t)(w_hi - w_lo) * 4, ctx.stream), ctx.detail);
      note_launch(), bpart_push_kernel<<<grid_for(2 * ps->words * 32, 256), 256, 0, ctx.stream>>>(
          push_adj(v, ps->dir), F, (uint32_t)(2 * ps->words), visited, ps->lo, ps->hi, N);
    } else {
      note_launch(), bpart_pull_kernel<<<grid_for((uint64_t)(w_hi - w_lo) * 32, 256), 256, 0,
                                         ctx.stream>>>(pull_adj(v, ps->dir), F, visited, ps->lo,
                                                       ps->hi, N);
    }
    note_launch(), bpart_settle_kernel<<<grid_for(w_hi - w_lo, 256), 256, 0, ctx.stream>>>(
        N, visited, ps->depth->as<uint32_t>(), ps->lo, ps->hi, level + 1, push_adj(v, ps->dir), acc);
    WC_CUDA(cudaGetLastError(), ctx.detail);
  }
  WC_TRY(ctx.finish());
  unsigned long long host[2];
  WC_CUDA(cudaMemcpy(host, acc, 16, cudaMemcpyDeviceToHost), ctx.detail);
  sums[0] = host[0];
  sums[1] = host[1];
  return WC_OK;
}

wc_status wc_bfs_part_end(wc_version* v, const wc_call* call, uint32_t* depth_out) {
  if (!v || !depth_out) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  PartSearch* ps = search_of(v);
  if (!ps) return WC_INVALID_ARGUMENT;
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ps->hi > ps->lo)
    WC_CUDA(cudaMemcpyAsync(depth_out + ps->lo, ps->depth->as<uint32_t>() + ps->lo,
                            (uint64_t)(ps->hi - ps->lo) * 4, cudaMemcpyDefault, ctx.stream),
            ctx.detail);
  const wc_status st = ctx.finish();
  {
    std::lock_guard<std::mutex> slock(g_searches_mu);
    g_searches.erase(v);  // the cuts stay with the version
  }
  return st;
}

}  // extern "C"
