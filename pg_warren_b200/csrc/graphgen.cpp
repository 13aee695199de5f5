// graphgen.cpp — deterministic synthetic graphs for the benchmarks and
// tests, built as the reference builds a version: rows sorted by target,
// parallel edges folded, self-loops dropped by the generator
// (graph/csr/build/deduplication.rs:1-79), and node ids relabelled through
// distinct random int64 external ids ranked in sorted order, the dense id
// being that rank (graph/id_map/mod.rs:38-49).
//
// R-MAT (Chakrabarti, Zhan, Faloutsos 2004): each edge descends `scale`
// levels of the adjacency matrix, choosing a quadrant with probabilities
// (a, b, c, 1-a-b-c).  Every random draw is a counter-based SplitMix64 of
// (seed, edge, level), so the graph does not depend on the thread count.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include "../../include/warren_cuda.h"

namespace {

constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ull;

inline uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// A uniform value in [0, 1) from 53 bits.
inline double unit(uint64_t bits) { return (double)(bits >> 11) * (1.0 / 9007199254740992.0); }

void parallel_for(uint64_t count, const std::function<void(uint64_t, uint64_t)>& body) {
  unsigned t = std::max(1u, std::thread::hardware_concurrency());
  if (count < (1u << 16)) t = 1;
  std::vector<std::thread> pool;
  uint64_t chunk = (count + t - 1) / t;
  for (unsigned w = 0; w < t; w++) {
    uint64_t lo = w * chunk, hi = std::min<uint64_t>(count, lo + chunk);
    if (lo >= hi) break;
    pool.emplace_back(body, lo, hi);
  }
  for (auto& th : pool) th.join();
}

// Relabels by ranks of distinct random external ids and builds the CSR:
// counting sort by source, then each row sorted and its repeats folded.
wc_status build(uint64_t n, std::vector<uint64_t>& src, std::vector<uint64_t>& dst, uint64_t seed,
                bool undirected, wc_host_csr* out) {
  // External ids: mix is a bijection of 64 bits, so they are distinct.
  std::vector<std::pair<int64_t, uint32_t>> ext(n);
  const uint64_t salt = mix(seed ^ 0x1d5eed1d5eedull);
  parallel_for(n, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; i++) ext[i] = {(int64_t)mix(salt + i * kGolden), (uint32_t)i};
  });
  std::sort(ext.begin(), ext.end());
  std::vector<uint32_t> dense(n);
  int64_t* external_ids = (int64_t*)malloc(std::max<uint64_t>(n, 1) * sizeof(int64_t));
  if (!external_ids) return WC_OUT_OF_MEMORY;
  for (uint64_t r = 0; r < n; r++) {
    dense[ext[r].second] = (uint32_t)r;
    external_ids[r] = ext[r].first;
  }
  const uint64_t raw = src.size();
  const uint64_t stored = undirected ? 2 * raw : raw;
  std::vector<uint64_t> deg(n + 1, 0);
  for (uint64_t e = 0; e < raw; e++) {
    deg[dense[src[e]] + 1]++;
    if (undirected) deg[dense[dst[e]] + 1]++;
  }
  for (uint64_t i = 0; i < n; i++) deg[i + 1] += deg[i];
  std::vector<uint32_t> tgt(stored);
  {
    std::vector<uint64_t> cur(deg.begin(), deg.end() - 1);
    for (uint64_t e = 0; e < raw; e++) {
      uint32_t s = dense[src[e]], t = dense[dst[e]];
      tgt[cur[s]++] = t;
      if (undirected) tgt[cur[t]++] = s;
    }
  }
  src.clear();
  src.shrink_to_fit();
  dst.clear();
  dst.shrink_to_fit();
  // Sort and fold each row (in place), counting what is kept.
  std::vector<uint64_t> kept(n, 0);
  parallel_for(n, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t r = lo; r < hi; r++) {
      uint32_t* b = tgt.data() + deg[r];
      uint32_t* e = tgt.data() + deg[r + 1];
      std::sort(b, e);
      kept[r] = std::unique(b, e) - b;
    }
  });
  uint64_t* offsets = (uint64_t*)malloc((n + 1) * sizeof(uint64_t));
  if (!offsets) {
    free(external_ids);
    return WC_OUT_OF_MEMORY;
  }
  offsets[0] = 0;
  for (uint64_t r = 0; r < n; r++) offsets[r + 1] = offsets[r] + kept[r];
  const uint64_t m = offsets[n];
  uint32_t* targets = (uint32_t*)malloc(std::max<uint64_t>(m, 1) * sizeof(uint32_t));
  if (!targets) {
    free(external_ids);
    free(offsets);
    return WC_OUT_OF_MEMORY;
  }
  parallel_for(n, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t r = lo; r < hi; r++)
      memcpy(targets + offsets[r], tgt.data() + deg[r], kept[r] * sizeof(uint32_t));
  });
  out->id_space = n;
  out->edges = m;
  out->offsets = offsets;
  out->targets = targets;
  out->external_ids = external_ids;
  return WC_OK;
}

}  // namespace

extern "C" {

wc_status wc_graph_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                        uint64_t seed, int32_t undirected, wc_host_csr* out) {
  if (!out || scale == 0 || scale > 31 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return WC_INVALID_ARGUMENT;
  memset(out, 0, sizeof *out);
  const uint64_t n = 1ull << scale;
  const uint64_t count = (uint64_t)edge_factor * n;
  std::vector<uint64_t> src(count), dst(count);
  std::vector<uint8_t> keep(count);
  const double ab = a + b, abc = a + b + c;
  const uint64_t key = mix(seed ^ kGolden);
  parallel_for(count, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t e = lo; e < hi; e++) {
      uint64_t s = 0, t = 0;
      const uint64_t base = mix(key + e * kGolden);
      for (uint32_t l = 0; l < scale; l++) {
        double u = unit(mix(base + (uint64_t)(l + 1) * 0xda942042e4dd58b5ull));
        uint64_t sb = u >= ab, tb = (u >= a && u < ab) || u >= abc;
        s = (s << 1) | sb;
        t = (t << 1) | tb;
      }
      src[e] = s;
      dst[e] = t;
      keep[e] = s != t;
    }
  });
  // Self-loops dropped.
  uint64_t w = 0;
  for (uint64_t e = 0; e < count; e++)
    if (keep[e]) {
      src[w] = src[e];
      dst[w] = dst[e];
      w++;
    }
  src.resize(w);
  dst.resize(w);
  return build(n, src, dst, seed, undirected != 0, out);
}

wc_status wc_graph_gnm(uint64_t n, uint64_t edges, uint64_t seed, int32_t undirected,
                       wc_host_csr* out) {
  if (!out || n == 0 || n >= (1ull << 32)) return WC_INVALID_ARGUMENT;
  memset(out, 0, sizeof *out);
  std::vector<uint64_t> src(edges), dst(edges);
  std::vector<uint8_t> keep(edges);
  const uint64_t key = mix(seed ^ 0x6e6d6e6d6e6dull);
  parallel_for(edges, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t e = lo; e < hi; e++) {
      uint64_t r = mix(key + e * kGolden);
      src[e] = (uint64_t)(((unsigned __int128)mix(r) * n) >> 64);
      dst[e] = (uint64_t)(((unsigned __int128)mix(r ^ kGolden) * n) >> 64);
      keep[e] = src[e] != dst[e];
    }
  });
  uint64_t w = 0;
  for (uint64_t e = 0; e < edges; e++)
    if (keep[e]) {
      src[w] = src[e];
      dst[w] = dst[e];
      w++;
    }
  src.resize(w);
  dst.resize(w);
  return build(n, src, dst, seed, undirected != 0, out);
}

void wc_host_csr_free(wc_host_csr* csr) {
  if (!csr) return;
  free(csr->offsets);
  free(csr->targets);
  free(csr->external_ids);
  memset(csr, 0, sizeof *csr);
}

}  // extern "C"
