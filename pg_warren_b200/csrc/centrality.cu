// centrality.cu — wc_centrality and wc_sample_sources: closeness and
// harmonic centrality (compute/centrality/closeness.rs:36-56) on unweighted
// rows, from every live node or from a seeded sample of them
// (centrality/sources.rs:55-123), run on the batched BFS.
//
// The sources go through the batched BFS in passes of up to 1,024 (whole
// 64-source batches, ascending); a pass keeps no depths but adds, for each
// node, how many of its sources first reach the node at each distance to
// the node's totals, in the order of the reference's batched measures
// (batch by batch, then by distance).  The reference searches without a
// depth limit: a pass runs 32 levels, and again with twice as many while
// its last level still had a frontier (up to 1,024).  The last kernel turns
// the totals into the reference's values (closeness.rs:117-132, 229-241).
#include <algorithm>
#include <queue>
#include <string>
#include <vector>

#include "batched.h"
#include "operand.h"

namespace wc {

constexpr uint32_t kCentStartLevels = 32;
constexpr uint32_t kCentMaxLevels = 1024;

__global__ void cent_fill_kernel(uint32_t* caps, uint32_t k, uint32_t levels) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x)
    caps[i] = levels;
}

__global__ void cent_sources_kernel(const uint64_t* sources, uint64_t count, uint32_t* is_source) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    atomicOr(is_source + (sources[i] >> 5), 1u << (sources[i] & 31));
}

// The values from the totals: `count` sources, `live` live nodes.
__global__ void cent_finish_kernel(uint32_t n, CentArgs c, const uint32_t* is_source,
                                   const uint64_t* tomb, uint64_t count, uint64_t live,
                                   uint32_t measure, bool wf_improved, double* values) {
  const bool every_live = count == live;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    double value = 0.0;
    const bool dead = tomb && ((tomb[u >> 6] >> (u & 63)) & 1);
    const uint64_t others = count - ((is_source[u >> 5] >> (u & 31)) & 1);
    if (!dead && measure == WC_CLOSENESS) {
      const double r = (double)c.reached[u];
      const double total = (double)c.dsum[u];
      if (total > 0.0 && live > 1) value = wf_improved ? r / total * (r / (double)others) : r / total;
    } else if (!dead) {
      const double total = c.harm[u];
      if (every_live) value = total;
      else if (others != 0) value = total * ((double)(live - 1) / (double)others);
    }
    values[u] = value;
  }
}

// The sampler's key of a node (sources.rs:121-123): SplitMix64's finaliser.
static uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
static uint64_t sample_key(uint64_t seed, uint64_t node) {
  return mix64(mix64(seed) ^ (node * 0x9e3779b97f4a7c15ull));
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_sample_sources(uint64_t id_space, const uint64_t* tombstone_words,
                            const uint8_t* population, int32_t complement, int64_t k,
                            uint64_t seed, uint64_t* sources_out, uint64_t* count_out) {
  if (!count_out || (id_space && !sources_out)) return WC_INVALID_ARGUMENT;
  // The population: live nodes the mask selects, ascending (sources.rs:55-79).
  std::vector<uint64_t> pop;
  for (uint64_t u = 0; u < id_space; u++) {
    const bool dead = tombstone_words && ((tombstone_words[u >> 6] >> (u & 63)) & 1);
    const bool selected = !population || ((population[u] != 0) != (complement != 0));
    if (selected && !dead) pop.push_back(u);
  }
  if (k >= 0 && (uint64_t)k < pop.size()) {
    // The k smallest keys (sources.rs:97-118), then ascending ids.
    std::priority_queue<std::pair<uint64_t, uint64_t>> largest;
    for (uint64_t u : pop) {
      const uint64_t key = sample_key(seed, u);
      if (largest.size() == (uint64_t)k) {
        if (k == 0 || key >= largest.top().first) continue;  // keys are distinct
        largest.pop();
      }
      largest.push({key, u});
    }
    pop.clear();
    for (; !largest.empty(); largest.pop()) pop.push_back(largest.top().second);
    std::sort(pop.begin(), pop.end());
  }
  std::copy(pop.begin(), pop.end(), sources_out);
  *count_out = pop.size();
  return WC_OK;
}

wc_status wc_centrality(wc_version* v, const wc_call* call, const wc_centrality_opts* o,
                        const uint64_t* sources, uint64_t count, const uint64_t* tombstone_words,
                        double* values_out) {
  if (!v || !o || (count && !sources) || (v->n && !values_out)) return WC_INVALID_ARGUMENT;
  if (o->measure != WC_CLOSENESS && o->measure != WC_HARMONIC) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  const uint64_t n = v->n;
  const uint64_t words = (n + 63) / 64;
  std::vector<uint64_t> tomb;
  if (tombstone_words) {
    tomb.resize(words);
    if (words)
      WC_CUDA(cudaMemcpy(tomb.data(), tombstone_words, words * 8, cudaMemcpyDefault), ctx.detail);
  }
  uint64_t live = n;
  for (uint64_t w : tomb) live -= __builtin_popcountll(w);
  std::vector<uint64_t> src(count);
  if (count)
    WC_CUDA(cudaMemcpy(src.data(), sources, count * 8, cudaMemcpyDefault), ctx.detail);
  // Sources: distinct live nodes, ascending (as the sampler gives them).
  for (uint64_t i = 0; i < count; i++) {
    if (src[i] >= n) {
      if (ctx.detail) ctx.detail->node = src[i];
      return WC_NODE_OUTSIDE_ID_SPACE;
    }
    if ((i && src[i] <= src[i - 1]) || (!tomb.empty() && ((tomb[src[i] >> 6] >> (src[i] & 63)) & 1))) {
      if (ctx.detail) ctx.detail->node = src[i];
      return WC_INVALID_ARGUMENT;
    }
  }
  uint32_t columns = o->columns_per_pass ? o->columns_per_pass : 1024;
  if (columns < 64 || columns > 1024 || (columns & (columns - 1))) return WC_INVALID_ARGUMENT;
  const uint32_t bps = o->blocks_per_sm ? o->blocks_per_sm : 4;
  WC_TRY(ctx.begin());
  if (n == 0) return ctx.finish();
  DevBuf *acc, *flag, *isrc, *capb, *srcb, *tb = nullptr;
  WC_TRY(ctx.scratch(POOL_CENT_TOTALS, n * 24, &acc));
  WC_TRY(ctx.scratch(POOL_CENT_FLAG, 16, &flag));
  WC_TRY(ctx.scratch(POOL_CENT_SOURCES, ((n + 31) / 32) * 4, &isrc));
  WC_TRY(ctx.scratch(POOL_CENT_CAPS, columns * 4, &capb));
  WC_TRY(ctx.scratch(POOL_CENT_LIST, std::max<uint64_t>(count, 1) * 8, &srcb));
  if (!tomb.empty()) {
    WC_TRY(ctx.scratch(POOL_CENT_TOMB, words * 8, &tb));
    WC_CUDA(cudaMemcpyAsync(tb->ptr, tomb.data(), words * 8, cudaMemcpyHostToDevice, ctx.stream),
            ctx.detail);
  }
  WC_CUDA(cudaMemsetAsync(acc->ptr, 0, n * 24, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(isrc->ptr, 0, ((n + 31) / 32) * 4, ctx.stream), ctx.detail);
  if (count)
    WC_CUDA(cudaMemcpyAsync(srcb->ptr, src.data(), count * 8, cudaMemcpyHostToDevice, ctx.stream),
            ctx.detail);
  CentArgs c;
  c.reached = acc->as<unsigned long long>();
  c.dsum = c.reached + n;
  c.harm = reinterpret_cast<double*>(c.dsum + n);
  c.cut = flag->as<int>();
  const uint64_t* sdev = srcb->as<uint64_t>();
  if (count)
    note_launch(), cent_sources_kernel<<<max_blocks(2), 256, 0, ctx.stream>>>(sdev, count,
                                                                          isrc->as<uint32_t>());
  // A search reaches every node it can within n - 1 levels.
  const uint32_t deepest = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(n - 1, 1), kCentMaxLevels);
  uint32_t levels = std::min(kCentStartLevels, deepest);
  BatchBuffers b;
  WC_TRY(b.reserve(ctx, columns / 32, levels));
  for (uint64_t s0 = 0; s0 < count;) {
    if (ctx.cancelled()) return ctx.finish();
    const uint32_t k = (uint32_t)std::min<uint64_t>(columns, count - s0);
    note_launch(), cent_fill_kernel<<<(k + 255) / 256, 256, 0, ctx.stream>>>(capb->as<uint32_t>(), k,
                                                                        levels);
    WC_CUDA(cudaMemsetAsync(c.cut, 0, 4, ctx.stream), ctx.detail);
    WC_TRY(bfs_centrality_pass(ctx, b, columns, sdev + s0, capb->as<uint32_t>(), k, levels, bps, c));
    int cut = 0;
    WC_CUDA(cudaMemcpyAsync(&cut, c.cut, 4, cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
    WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
    if (levels >= n - 1) cut = 0;  // nothing lies deeper than n - 1 levels
    if (cut && levels < deepest) {
      // The totals were left as they were: the pass runs again, deeper.
      levels = std::min(2 * levels, deepest);
      WC_TRY(b.reserve(ctx, columns / 32, levels));
      continue;
    }
    if (cut) {
      if (ctx.detail)
        snprintf(ctx.detail->message, sizeof ctx.detail->message,
                 "a search runs deeper than %u levels", kCentMaxLevels);
      return WC_UNSUPPORTED;
    }
    ctx.progress("centrality", s0 + k, count);
    s0 += k;
  }
  Operand out(POOL_CENT_VALUES);
  WC_TRY(out.output(ctx, values_out, n * 8));
  note_launch(), cent_finish_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(
      (uint32_t)n, c, isrc->as<uint32_t>(), tb ? tb->as<uint64_t>() : nullptr, count, live,
      o->measure, o->wf_improved != 0, static_cast<double*>(out.dev));
  WC_TRY(out.out(ctx));
  return ctx.finish();
}

}  // extern "C"
