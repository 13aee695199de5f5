// betweenness.cu — wc_betweenness: betweenness centrality by Brandes'
// algorithm on unweighted rows (compute/centrality/betweenness.rs:27-110,
// paths.rs:148-260), from every live node or from sampled sources, rescaled
// as betweenness.rs:113-141 rescales.
//
// The sources run 64 at a time through the batched BFS, which keeps one
// frontier snapshot per level: bit s of node v's row of F_L says that
// source s first reaches v at distance L.  Then, per level, on the device,
// over the row-split schedules (long rows in pieces of 256 entries):
//  - path counts σ (f64, n × 64): a node first reached at L sums σ over
//    its in-neighbours at L - 1.  The counts are integers, exact in f64 up
//    to 2^53, so their order does not matter;
//  - dependencies δ, from the deepest level up: δ(v) = Σ σ(v)/σ(w) ·
//    (1 + δ(w)) over v's out-neighbours w one level further, taken in
//    ascending order, term by term, as paths.rs:244-260 takes them (rows
//    over 256 entries: each piece in order, then the pieces in order);
//  - then each node's total gains the pass's 64 sources' dependencies in
//    source order (betweenness.rs:76-93 folds sources in ascending order).
// Up to the path counts' 2^53 and rows over 256 entries, the values are the
// reference's to the bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "batched.h"
#include "operand.h"

namespace wc {

constexpr uint32_t kBcColumns = 64;  // sources a pass
constexpr int kBcWords = 2;          // their frontier words
constexpr uint32_t kBcStartLevels = 32;
constexpr uint32_t kBcMaxLevels = 1024;

struct BcPass {
  uint32_t n;
  uint64_t fstride;        // words between snapshots
  const uint32_t* F;       // snapshots, rows of kBcWords words
  const uint32_t* wbits;   // per level: the rows written
  uint32_t bitmap_words;
  const uint32_t* roff;    // reverse CSR (in-neighbours)
  const uint32_t* rtgt;
  const uint32_t* foff;    // forward CSR (out-neighbours)
  const uint32_t* ftgt;
  const Unit* runits;      // the reverse CSR's row-split schedule
  uint32_t rcount;
  const Unit* funits;      // the forward CSR's, with its long rows' counters
  uint32_t fcount;
  uint32_t* counters;      // left zero
  double* carry;           // slots × 64: the forward long rows' piece sums
  double* sigma;           // n × 64
  double* delta;           // n × 64
};

__device__ inline bool written(const BcPass& P, uint32_t L, uint32_t v) {
  return (P.wbits[(size_t)L * P.bitmap_words + (v >> 5)] >> (v & 31)) & 1;
}
__device__ inline uint32_t row_word(const BcPass& P, uint32_t L, uint32_t v, int q) {
  return P.F[(size_t)L * P.fstride + (size_t)v * kBcWords + q];
}

__global__ void bc_seed_kernel(const uint64_t* sources, uint32_t k, double* sigma) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < k) sigma[sources[s] * kBcColumns + s] = 1.0;
}

// The σ sum of one row's entries [e0, e1) for this lane's sources: the
// in-neighbours u at level L - 1 whose bit is set.
__device__ inline void sigma_run(const BcPass& P, uint32_t L, uint32_t e0, uint32_t e1,
                                 const bool (&mine)[kBcWords], double (&acc)[kBcWords]) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t e = e0; e < e1; e++) {
    const uint32_t u = P.rtgt[e];
    if (!written(P, L - 1, u)) continue;
#pragma unroll
    for (int q = 0; q < kBcWords; q++)
      if (mine[q] && ((row_word(P, L - 1, u, q) >> lane) & 1))
        acc[q] += P.sigma[(size_t)u * kBcColumns + 32 * q + lane];
  }
}

// σ of the rows first reached at level L (L >= 1), over the reverse CSR's
// row-split schedule: a warp per unit, lane `lane` for sources lane and
// 32 + lane.  A tile's rows are summed whole; a long row's pieces add their
// sums atomically (path counts are integers: the order cannot change them).
__global__ void bc_sigma_kernel(BcPass P, uint32_t L) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < P.rcount; u += warps) {
    const Unit U = P.runits[u];
    const bool tile = (U.c >> 31) == 0;
    const uint32_t r0 = U.a, r1 = tile ? U.b : U.a + 1;
    for (uint32_t v = r0; v < r1; v++) {
      if (!written(P, L, v)) continue;
      bool mine[kBcWords];
      double acc[kBcWords];
#pragma unroll
      for (int q = 0; q < kBcWords; q++) {
        mine[q] = (row_word(P, L, v, q) >> lane) & 1;
        acc[q] = 0.0;
      }
      if (tile) {
        sigma_run(P, L, P.roff[v], P.roff[v + 1], mine, acc);
#pragma unroll
        for (int q = 0; q < kBcWords; q++)
          if (mine[q]) P.sigma[(size_t)v * kBcColumns + 32 * q + lane] = acc[q];
      } else {
        sigma_run(P, L, U.b, U.d, mine, acc);
#pragma unroll
        for (int q = 0; q < kBcWords; q++)
          if (mine[q] && acc[q] != 0.0)
            atomicAdd(P.sigma + (size_t)v * kBcColumns + 32 * q + lane, acc[q]);
      }
    }
  }
}

// The dependency terms of one row's entries [e0, e1), in order, added to
// `gained`: σ(v)/σ(w) · (1 + δ(w)) over the out-neighbours w one level on.
__device__ inline void delta_run(const BcPass& P, uint32_t L, uint32_t e0, uint32_t e1,
                                 const bool (&mine)[kBcWords], const double (&sv)[kBcWords],
                                 double (&gained)[kBcWords]) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t e = e0; e < e1; e++) {
    const uint32_t w = P.ftgt[e];
    if (!written(P, L + 1, w)) continue;
#pragma unroll
    for (int q = 0; q < kBcWords; q++)
      if (mine[q] && ((row_word(P, L + 1, w, q) >> lane) & 1)) {
        const size_t at = (size_t)w * kBcColumns + 32 * q + lane;
        gained[q] += sv[q] / P.sigma[at] * (1.0 + P.delta[at]);
      }
  }
}

// δ of the rows first reached at level L, from level L + 1's (already
// final), over the forward CSR's schedule: a tile's rows in order, term by
// term (paths.rs:244-260); a long row's pieces each in order, then the
// pieces' sums in piece order by the warp that brings the last piece, so
// only rows over 256 entries are reassociated.
__global__ void bc_delta_kernel(BcPass P, uint32_t L) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < P.fcount; u += warps) {
    const Unit U = P.funits[u];
    const bool tile = (U.c >> 31) == 0;
    const uint32_t r0 = U.a, r1 = tile ? U.b : U.a + 1;
    for (uint32_t v = r0; v < r1; v++) {
      if (!written(P, L, v)) continue;
      bool mine[kBcWords];
      double sv[kBcWords], gained[kBcWords];
#pragma unroll
      for (int q = 0; q < kBcWords; q++) {
        mine[q] = (row_word(P, L, v, q) >> lane) & 1;
        sv[q] = mine[q] ? P.sigma[(size_t)v * kBcColumns + 32 * q + lane] : 0.0;
        gained[q] = 0.0;
      }
      if (tile) {
        delta_run(P, L, P.foff[v], P.foff[v + 1], mine, sv, gained);
#pragma unroll
        for (int q = 0; q < kBcWords; q++)
          if (mine[q]) P.delta[(size_t)v * kBcColumns + 32 * q + lane] = gained[q];
        continue;
      }
      delta_run(P, L, U.b, U.d, mine, sv, gained);
      const uint32_t slot = U.c & 0x7fffffffu;
      const uint32_t row_lo = P.foff[v], deg = P.foff[v + 1] - row_lo;
      const uint32_t pieces = (deg + kPieceEntries - 1) / kPieceEntries;
      const uint32_t first = slot - (U.b - row_lo) / kPieceEntries;
#pragma unroll
      for (int q = 0; q < kBcWords; q++) P.carry[(size_t)slot * kBcColumns + 32 * q + lane] = gained[q];
      __threadfence();
      __syncwarp();
      uint32_t arrived = 0;
      if (lane == 0) arrived = atomicAdd(P.counters + first, 1u);
      arrived = __shfl_sync(0xffffffffu, arrived, 0);
      if (arrived == pieces - 1) {
        __threadfence();
#pragma unroll
        for (int q = 0; q < kBcWords; q++) {
          double total = 0.0;
          for (uint32_t p = 0; p < pieces; p++)
            total += __ldcg(P.carry + (size_t)(first + p) * kBcColumns + 32 * q + lane);
          if (mine[q]) P.delta[(size_t)v * kBcColumns + 32 * q + lane] = total;
        }
        __syncwarp();
        if (lane == 0) P.counters[first] = 0;
      }
    }
  }
}

// The nodes each source reaches (σ > 0), for endpoints.
__global__ void bc_reached_kernel(const double* sigma, uint32_t n, unsigned long long* reached) {
  __shared__ unsigned counts[kBcColumns];
  for (uint32_t s = threadIdx.x; s < kBcColumns; s += blockDim.x) counts[s] = 0;
  __syncthreads();
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < (uint64_t)n * kBcColumns;
       x += (uint64_t)gridDim.x * blockDim.x)
    if (sigma[x] > 0.0) atomicAdd(&counts[x % kBcColumns], 1u);
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < kBcColumns; s += blockDim.x)
    if (counts[s]) atomicAdd(reached + s, (unsigned long long)counts[s]);
}

// Each node's total gains the pass's sources' dependencies, in source
// order; a source gains nothing on its own search, or with endpoints the
// number of other nodes it reaches, and with endpoints every node it
// reaches gains one more (betweenness.rs:55-71).
__global__ void bc_fold_kernel(const double* sigma, const double* delta, const uint64_t* sources,
                               uint32_t k, uint32_t n, bool endpoints,
                               const unsigned long long* reached, double* total) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    double t = total[v];
    for (uint32_t s = 0; s < k; s++) {
      const size_t at = (size_t)v * kBcColumns + s;
      double g;
      if (sources[s] == v) {
        g = endpoints ? (double)(reached[s] - 1) : 0.0;
      } else {
        g = delta[at];
        if (endpoints && sigma[at] > 0.0) g += 1.0;
      }
      t += g;
    }
    total[v] = t;
  }
}

// betweenness.rs:95-110: the source factor for sampled sources, the other
// factor for every other node; tombstoned nodes 0.
__global__ void bc_finish_kernel(const double* total, uint32_t n, const uint32_t* is_source,
                                 const uint64_t* tomb, double source_factor, double other_factor,
                                 double* values) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const bool dead = tomb && ((tomb[v >> 6] >> (v & 63)) & 1);
    const bool src = is_source && ((is_source[v >> 5] >> (v & 31)) & 1);
    values[v] = dead ? 0.0 : total[v] * (src ? source_factor : other_factor);
  }
}

__global__ void bc_sources_kernel(const uint64_t* sources, uint64_t count, uint32_t* is_source) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    atomicOr(is_source + (sources[i] >> 5), 1u << (sources[i] & 31));
}

__global__ void bc_fill_kernel(uint32_t* caps, uint32_t k, uint32_t levels) {
  for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) caps[i] = levels;
}

// betweenness.rs:113-141 (rescale) for n live nodes and k sampled sources
// (every live node: k < 0).
static void rescale(uint64_t n, bool normalized, bool endpoints, bool directed, int64_t k,
                    double* source_factor, double* other_factor) {
  const __int128 pairs = (__int128)n - (endpoints ? 0 : 1);
  if (pairs < 2) {
    *source_factor = *other_factor = 1.0;
    return;
  }
  const __int128 correction = directed ? 1 : 2;
  const __int128 k_sources = k < 0 ? pairs : k;
  auto factor = [&](__int128 sources) {
    return normalized ? 1.0 / (double)(sources * (pairs - 1))
                      : (double)pairs / (double)(sources * correction);
  };
  if (k < 0 || endpoints) {
    *source_factor = *other_factor = factor(k_sources);
  } else {
    *source_factor = k_sources > 1 ? factor(k_sources - 1) : NAN;
    *other_factor = factor(k_sources);
  }
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_betweenness(wc_version* v, const wc_call* call, const wc_betweenness_opts* o,
                         const uint64_t* sources, uint64_t count, const uint64_t* tombstone_words,
                         double* values_out) {
  if (!v || !o || (count && !sources) || (v->n && !values_out)) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  const uint64_t n = v->n;
  const uint64_t words = (n + 63) / 64;
  std::vector<uint64_t> tomb;
  if (tombstone_words && words) {
    tomb.resize(words);
    WC_CUDA(cudaMemcpy(tomb.data(), tombstone_words, words * 8, cudaMemcpyDefault), ctx.detail);
  }
  uint64_t live = n;
  for (uint64_t w : tomb) live -= __builtin_popcountll(w);
  std::vector<uint64_t> src(count);
  if (count)
    WC_CUDA(cudaMemcpy(src.data(), sources, count * 8, cudaMemcpyDefault), ctx.detail);
  for (uint64_t i = 0; i < count; i++) {  // distinct live nodes, ascending
    if (src[i] >= n) {
      if (ctx.detail) ctx.detail->node = src[i];
      return WC_NODE_OUTSIDE_ID_SPACE;
    }
    if ((i && src[i] <= src[i - 1]) || (!tomb.empty() && ((tomb[src[i] >> 6] >> (src[i] & 63)) & 1))) {
      if (ctx.detail) ctx.detail->node = src[i];
      return WC_INVALID_ARGUMENT;
    }
  }
  const uint32_t bps = o->blocks_per_sm ? o->blocks_per_sm : 4;
  WC_TRY(ctx.begin());
  if (n == 0) return ctx.finish();
  const bool every_live = count == live;
  double source_factor, other_factor;
  rescale(live, o->normalized != 0, o->endpoints != 0, o->directed != 0,
          every_live ? -1 : (int64_t)count, &source_factor, &other_factor);
  DevBuf *sig, *del, *tot, *rch, *flag, *isrc, *capb, *srcb, *tb = nullptr;
  WC_TRY(ctx.scratch(POOL_BC_SIGMA, n * kBcColumns * 8, &sig));
  WC_TRY(ctx.scratch(POOL_BC_DELTA, n * kBcColumns * 8, &del));
  WC_TRY(ctx.scratch(POOL_BC_TOTAL, n * 8, &tot));
  WC_TRY(ctx.scratch(POOL_BC_REACHED, kBcColumns * 8, &rch));
  WC_TRY(ctx.scratch(POOL_BC_FLAG, 16, &flag));
  WC_TRY(ctx.scratch(POOL_BC_SOURCES, ((n + 31) / 32) * 4, &isrc));
  WC_TRY(ctx.scratch(POOL_BC_CAPS, kBcColumns * 4, &capb));
  WC_TRY(ctx.scratch(POOL_BC_LIST, std::max<uint64_t>(count, 1) * 8, &srcb));
  DevBuf* carry;
  WC_TRY(ctx.scratch(POOL_BC_CARRY,
                     (uint64_t)std::max<uint32_t>(v->fwd.schedule.slots, 1) * kBcColumns * 8, &carry));
  if (!tomb.empty()) {
    WC_TRY(ctx.scratch(POOL_BC_TOMB, words * 8, &tb));
    WC_CUDA(cudaMemcpyAsync(tb->ptr, tomb.data(), words * 8, cudaMemcpyHostToDevice, ctx.stream),
            ctx.detail);
  }
  WC_CUDA(cudaMemsetAsync(tot->ptr, 0, n * 8, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(isrc->ptr, 0, ((n + 31) / 32) * 4, ctx.stream), ctx.detail);
  if (count)
    WC_CUDA(cudaMemcpyAsync(srcb->ptr, src.data(), count * 8, cudaMemcpyHostToDevice, ctx.stream),
            ctx.detail);
  const uint64_t* sdev = srcb->as<uint64_t>();
  if (count && !every_live)
    note_launch(), bc_sources_kernel<<<max_blocks(2), 256, 0, ctx.stream>>>(sdev, count,
                                                                        isrc->as<uint32_t>());
  CentArgs c{};
  c.cut = flag->as<int>();
  c.keep_only = true;
  const uint32_t deepest = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(n - 1, 1), kBcMaxLevels);
  uint32_t levels = std::min(kBcStartLevels, deepest);
  BatchBuffers b;
  WC_TRY(b.reserve(ctx, kBcWords, levels));
  const uint32_t bitmap_words = (uint32_t)((n + 31) / 32);
  const uint32_t grid = max_blocks((int)bps);
  for (uint64_t s0 = 0; s0 < count;) {
    if (ctx.cancelled()) return ctx.finish();
    const uint32_t k = (uint32_t)std::min<uint64_t>(kBcColumns, count - s0);
    note_launch(), bc_fill_kernel<<<1, 64, 0, ctx.stream>>>(capb->as<uint32_t>(), k, levels);
    WC_CUDA(cudaMemsetAsync(c.cut, 0, 4, ctx.stream), ctx.detail);
    WC_TRY(bfs_centrality_pass(ctx, b, kBcColumns, sdev + s0, capb->as<uint32_t>(), k, levels, bps,
                               c));
    int cut = 0;
    WC_CUDA(cudaMemcpyAsync(&cut, c.cut, 4, cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
    WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
    if (levels >= n - 1) cut = 0;  // nothing lies deeper than n - 1 levels
    if (cut && levels < deepest) {
      levels = std::min(2 * levels, deepest);
      WC_TRY(b.reserve(ctx, kBcWords, levels));
      continue;
    }
    if (cut) {
      set_message(ctx.detail, "a search runs deeper than %u levels", kBcMaxLevels);
      return WC_UNSUPPORTED;
    }
    // The snapshots: F_L at L · n · 2 words, the written-row maps after the
    // frontier maps (BatchBuffers::reserve).
    const uint64_t maps = (uint64_t)(levels + 2) * bitmap_words;
    BcPass P{(uint32_t)n, n * kBcWords, b.F->as<uint32_t>(), b.bits->as<uint32_t>() + maps,
             bitmap_words, v->rev.offsets.as<uint32_t>(), v->rev.targets.as<uint32_t>(),
             v->fwd.offsets.as<uint32_t>(), v->fwd.targets.as<uint32_t>(),
             v->rev.schedule.units.as<Unit>(), v->rev.schedule.count,
             v->fwd.schedule.units.as<Unit>(), v->fwd.schedule.count,
             v->fwd.schedule.counters.as<uint32_t>(), carry->as<double>(), sig->as<double>(),
             del->as<double>()};
    WC_CUDA(cudaMemsetAsync(sig->ptr, 0, n * kBcColumns * 8, ctx.stream), ctx.detail);
    WC_CUDA(cudaMemsetAsync(del->ptr, 0, n * kBcColumns * 8, ctx.stream), ctx.detail);
    note_launch(), bc_seed_kernel<<<1, 64, 0, ctx.stream>>>(sdev + s0, k, sig->as<double>());
    for (uint32_t L = 1; L <= levels; L++)
      note_launch(), bc_sigma_kernel<<<grid, 256, 0, ctx.stream>>>(P, L);
    for (uint32_t L = levels; L-- > 0;)
      note_launch(), bc_delta_kernel<<<grid, 256, 0, ctx.stream>>>(P, L);
    if (o->endpoints) {
      WC_CUDA(cudaMemsetAsync(rch->ptr, 0, kBcColumns * 8, ctx.stream), ctx.detail);
      note_launch(), bc_reached_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(
          sig->as<double>(), (uint32_t)n, rch->as<unsigned long long>());
    }
    note_launch(), bc_fold_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(
        sig->as<double>(), del->as<double>(), sdev + s0, k, (uint32_t)n, o->endpoints != 0,
        rch->as<unsigned long long>(), tot->as<double>());
    ctx.progress("betweenness", s0 + k, count);
    s0 += k;
  }
  Operand out(POOL_BC_VALUES);
  WC_TRY(out.output(ctx, values_out, n * 8));
  note_launch(), bc_finish_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(
      tot->as<double>(), (uint32_t)n, every_live ? nullptr : isrc->as<uint32_t>(),
      tb ? tb->as<uint64_t>() : nullptr, source_factor, other_factor,
      static_cast<double*>(out.dev));
  WC_TRY(out.out(ctx));
  return ctx.finish();
}

}  // extern "C"
