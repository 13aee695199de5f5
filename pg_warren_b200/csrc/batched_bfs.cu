// batched_bfs.cu — wc_bfs_batched and wc_autotune: many BFS searches as one
// boolean SpMM over bit-packed frontiers (no reference counterpart; its CPU
// prior art is compute/centrality/multi_source.rs, 64 sources per word).
//
// A pass takes up to 1,024 sources, one bit each in a row of W 32-bit words
// per node (W = columns / 32).  Level L pulls over the reverse CSR: node i
// ORs the frontier rows F_L[j] of its in-neighbours j (only those whose row
// is non-zero for a source still expanding, read from a frontier bitmap),
// keeps the bits it has not seen, and writes them as its row of F_{L+1}.  A
// source with depth cap c expands levels 0 .. c-1, as the reference's
// LevelSearch stops at max_depth (traversal/level.rs:119-123), so its bits
// are masked out of the frontier from level c on.  Every F_L is kept (the
// kernel writes each row, new bits or zero), and a last kernel turns them
// into per-source depths, source-major, while summing the out-degree of each
// node a source expands: the row entries a push-only bfs from that source
// scans (its edges_traversed).
//
// Every level's launches are queued without a host round trip: a level whose
// frontier is empty returns at once, reading the count the previous level
// wrote.  The pass is therefore a fixed launch sequence, captured once per
// (version, pass shape) into a CUDA graph and replayed.
#include <algorithm>
#include <string>

#include "batched.h"
#include "operand.h"
#include "semiring.cuh"

namespace wc {

__device__ inline bool nbit(const uint32_t* b, uint32_t i) { return (b[i >> 5] >> (i & 31)) & 1; }

// Zeroes the sources' rows of F_0 (the only rows of F_0 that are read).
template <int W>
__global__ void msbfs_clear_kernel(const uint64_t* sources, uint32_t k, uint32_t* F0) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < k) {
    uint32_t* row = F0 + (size_t)sources[t] * W;
    for (int w = 0; w < W; w++) row[w] = 0;
  }
}

// Seeds: F_0 and V get bit s at node sources[s] (F_0's rows are marked
// written); every source is live at level 0; the level masks A_L (bits of
// sources with cap > L) are built for every level.
template <int W>
__global__ void msbfs_seed_kernel(const uint64_t* sources, const uint32_t* caps, uint32_t k,
                                  uint32_t levels, uint32_t n, uint32_t* V, uint32_t* F0,
                                  uint32_t* fbits0, uint32_t* wbits0, uint32_t* masks,
                                  uint32_t* alive0, uint32_t* counts, const uint32_t* foff,
                                  unsigned long long* fedges0) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < k) {
    const uint32_t node = (uint32_t)sources[t];
    atomicOr(V + (size_t)node * W + (t >> 5), 1u << (t & 31));
    atomicOr(F0 + (size_t)node * W + (t >> 5), 1u << (t & 31));
    atomicOr(wbits0 + (node >> 5), 1u << (node & 31));
    atomicOr(alive0 + (t >> 5), 1u << (t & 31));
    if (caps[t] > 0) {
      atomicOr(fbits0 + (node >> 5), 1u << (node & 31));
      atomicAdd(fedges0, (unsigned long long)(foff[node + 1] - foff[node]));
    }
  }
  // masks[L * W + w]: bit b set if source 32w+b exists and cap > L.
  for (uint32_t x = t; x < levels * W; x += gridDim.x * blockDim.x) {
    const uint32_t L = x / W, w = x % W;
    uint32_t m = 0;
    for (uint32_t b = 0; b < 32; b++) {
      const uint32_t s = 32 * w + b;
      if (s < k && caps[s] > L) m |= 1u << b;
    }
    masks[x] = m;
  }
  if (t == 0) counts[0] = 1;  // level 0's frontier is non-empty (or harmlessly so)
}

// Level L: F_{L+1}[i] = (OR over in-neighbours j in the frontier of
// F_L[j] & A_L) & ~V[i]; V[i] |= F_{L+1}[i].  Warps walk the reverse CSR's
// row-split schedule (units of at most 256 entries).  In a tile of rows the
// warp first finds which rows still lack a source (the rest are skipped),
// loads the tile's targets and their frontier bits with eight loads in
// flight a lane, lists the hits, then gathers the hit rows of F_L, several
// at once, OR-ing them into per-row accumulators in shared memory.  A long
// row's pieces OR into a per-row accumulator in global memory, and the last
// piece to arrive writes the row.
struct MsLevel {
  uint32_t n;
  const uint32_t* off;
  const uint32_t* tgt;
  const Unit* units;
  uint32_t unit_count;
  uint32_t* counters;  // per long row (first slot), left zero
  uint32_t* nacc;      // W words per long row (first slot), left zero
  uint32_t* V;
  const uint32_t* Fcur;
  uint32_t* Fnext;
  const uint32_t* fbits;
  uint32_t* fbits_next;
  uint32_t* wbits_next;  // rows of F_{L+1} written (the others are zero)
  const uint32_t* masks;
  uint32_t* alive;       // [level][W]: sources with a non-empty frontier
  uint32_t L;
  uint32_t* counts;
  unsigned long long* fedges;  // [level]: out-edges of the rows expanding there
  const uint32_t* foff;        // the forward CSR (push levels, out-degrees)
  const uint32_t* ftgt;
  const Unit* funits;
  uint32_t funit_count;
  uint64_t m;
  uint32_t* acc;      // n × W push accumulators, all zero between levels
  uint32_t* touched;  // rows with a push accumulator to settle, all zero between levels
  uint32_t* pulled;   // if set: counts the levels that pull (timed calls)
  const uint32_t* unit_rows;  // per unit of `units`: its rows that hold entries
};

// Whether level P.L runs at all: it has a frontier.  A level that does not
// run leaves the next level's count zero, so every later level returns at
// once too.
__device__ inline bool level_runs(const MsLevel& P) { return P.counts[P.L] != 0; }

// Before each level's kernels: a raised cancel word (host-mapped, read here
// by one thread) empties the level's frontier count, so all of the level's
// kernels and every later level return at once.  The count changes only
// between kernels, so a level runs whole or not at all, and the buffers kept
// zero between calls stay zero.
__global__ void msbfs_cancel_kernel(const int32_t* cancel, uint32_t* count) {
  if (threadIdx.x == 0 && *(volatile const int32_t*)cancel) *count = 0;
}

// A level pushes (scatters the frontier rows over the forward CSR) while the
// frontier's out-edges are below m / kPushDivisor, and pulls (gathers over
// the reverse CSR) otherwise; every kernel of the level reads the same
// counts, so they agree on the choice.
constexpr uint64_t kPushDivisor = 32;
__device__ inline bool level_pushes(const MsLevel& P) {
  return P.fedges[P.L] * kPushDivisor < P.m;
}

// A warp's contribution to the next level's counts: rows admitted, their
// out-edges, and the live sources.
template <int W>
__device__ inline void level_totals(const MsLevel& P, uint32_t admitted, unsigned long long fed,
                                    uint32_t live) {
  const unsigned lane = threadIdx.x & 31;
  for (int o = 16; o > 0; o >>= 1) {
    admitted += __shfl_down_sync(0xffffffffu, admitted, o);
    fed += __shfl_down_sync(0xffffffffu, fed, o);
  }
  if (lane == 0 && admitted) {
    atomicAdd(P.counts + P.L + 1, admitted);
    atomicAdd(P.fedges + P.L + 1, fed);
  }
#pragma unroll
  for (uint32_t o = W; o < 32; o <<= 1) live |= __shfl_xor_sync(0xffffffffu, live, o);
  if (lane < W && live) atomicOr(P.alive + (P.L + 1) * W + lane, live);
}

template <int W> struct MsWarpSmem {
  uint32_t acc[32 * W];
  uint32_t hitj[kTileEntries];
  uint8_t hitr[kTileEntries];
  uint8_t rowof[kTileEntries];  // the tile row of each entry
};

// A lane's VEC consecutive words of a row, moved with one vector access.
template <int N> struct Words {
  uint32_t x[N];
};
template <int N> __device__ inline Words<N> load_words(const uint32_t* p) {
  Words<N> r;
  if constexpr (N == 4) {
    const uint4 v = *reinterpret_cast<const uint4*>(p);
    r.x[0] = v.x; r.x[1] = v.y; r.x[2] = v.z; r.x[3] = v.w;
  } else if constexpr (N == 2) {
    const uint2 v = *reinterpret_cast<const uint2*>(p);
    r.x[0] = v.x; r.x[1] = v.y;
  } else {
    r.x[0] = *p;
  }
  return r;
}
template <int N> __device__ inline Words<N> ldg_words(const uint32_t* p) {
  Words<N> r;
  if constexpr (N == 4) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    r.x[0] = v.x; r.x[1] = v.y; r.x[2] = v.z; r.x[3] = v.w;
  } else if constexpr (N == 2) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
    r.x[0] = v.x; r.x[1] = v.y;
  } else {
    r.x[0] = __ldg(p);
  }
  return r;
}
template <int N> __device__ inline void store_words(uint32_t* p, const Words<N>& r) {
  if constexpr (N == 4) *reinterpret_cast<uint4*>(p) = make_uint4(r.x[0], r.x[1], r.x[2], r.x[3]);
  else if constexpr (N == 2) *reinterpret_cast<uint2*>(p) = make_uint2(r.x[0], r.x[1]);
  else *p = r.x[0];
}
template <int N> __device__ inline bool any_words(const Words<N>& r) {
  uint32_t o = 0;
#pragma unroll
  for (int i = 0; i < N; i++) o |= r.x[i];
  return o != 0;
}

// Requests into L2 the lines a unit reads first — its rows' visited words,
// its targets and (a tile) its row offsets — so that when the warp reaches
// the unit those loads hit L2 rather than DRAM.  Every address is inside
// the unit's own ranges.
__device__ inline void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
template <int W>
__device__ inline void prefetch_unit(const MsLevel& P, const Unit& d, uint32_t held,
                                     unsigned lane) {
  const bool tile = (d.c >> 31) == 0;
  const uint32_t r0 = d.a, R = tile ? d.b - d.a : 1;
  const uint32_t e0 = tile ? d.d : d.b, cnt = tile ? d.c : d.d - d.b;
  if (lane < R && ((held >> lane) & 1)) prefetch_l2(P.V + (size_t)(r0 + lane) * W);
  if (32 * lane < cnt) prefetch_l2(P.tgt + e0 + 32 * lane);
  if (tile && lane == 31) prefetch_l2(P.off + r0);
}

// The pull of one level.  A row's W words are spread over LPR = W/VEC
// lanes holding VEC words each (one 16-byte access for W >= 4), so a warp
// instruction covers G = 32/LPR rows or gathered frontier rows.  While a
// unit runs, the warp's next unit is prefetched into L2 (its descriptor
// was loaded one unit earlier, so the prefetch does not wait on it).
template <int W>
__global__ void __launch_bounds__(256, 4) msbfs_level_kernel(MsLevel P) {
  if (!level_runs(P)) return;  // nothing expands (or cancelled): F_{L+1} is not read
  if (level_pushes(P)) return;  // msbfs_push_kernel and msbfs_settle_kernel run it
  if (P.pulled && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(P.pulled, 1u);
  constexpr uint32_t VEC = W >= 4 ? 4 : W;
  constexpr uint32_t LPR = W / VEC;
  constexpr uint32_t G = 32 / LPR;
  constexpr uint32_t GM = LPR == 32 ? 0xffffffffu : (1u << LPR) - 1;
  constexpr int Q = kTileEntries / 32;
  constexpr int U = 8;  // frontier rows in flight per lane
  using V4 = Words<VEC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MsWarpSmem<W>& sm = reinterpret_cast<MsWarpSmem<W>*>(smem_raw)[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31;
  const unsigned sub = lane / LPR, q = lane % LPR;
  const uint32_t w0 = q * VEC;
  const unsigned gmask = GM << (sub * LPR);
  // Sources still searching: cap above L and a non-empty frontier.  A row
  // all of whose such sources have reached it needs nothing this level.
  V4 a = load_words<VEC>(P.masks + P.L * W + w0);
  {
    const V4 alive = load_words<VEC>(P.alive + P.L * W + w0);
#pragma unroll
    for (int i = 0; i < (int)VEC; i++) a.x[i] &= alive.x[i];
  }
  // The next level's searching sources are read where a row is written
  // (an L1 hit), not kept in registers across the gathers.
  const uint32_t* a_next_p = P.masks + (P.L + 1) * W + w0;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  uint32_t admitted = 0;
  unsigned long long fed = 0;  // out-edges of the rows admitted
  V4 live = {};                // this warp's fresh bits, for the next level's live set

  Unit nxt{};
  uint32_t nxt_held = 0;
  if (warp + warps < P.unit_count) {
    nxt = P.units[warp + warps];
    nxt_held = P.unit_rows[warp + warps];
  }
  for (uint32_t u = warp; u < P.unit_count; u += warps) {
    const Unit unit = P.units[u];  // loaded a unit earlier as `nxt`: a cache hit
    // The rows that hold entries: a row with none (about half of an R-MAT
    // graph's) can gain no bits, so its visited words are not read.
    const uint32_t held = P.unit_rows[u];
    if (u + warps < P.unit_count) {
      prefetch_unit<W>(P, nxt, nxt_held, lane);
      if (u + 2 * warps < P.unit_count) {
        nxt = P.units[u + 2 * warps];
        nxt_held = P.unit_rows[u + 2 * warps];
      }
    }
    const bool tile = (unit.c >> 31) == 0;
    const uint32_t r0 = unit.a;
    const uint32_t R = tile ? unit.b - unit.a : 1;
    // Which rows still lack a searching source: the rows' V words are all
    // loaded first (kept for the write at the end), then tested.
    constexpr uint32_t VR = kTileRows / G > 0 ? kTileRows / G : 1;
    V4 vrow[VR];
#pragma unroll
    for (uint32_t x = 0; x < VR; x++) {
      const uint32_t r = x * G + sub;
      if (r < R && ((held >> r) & 1)) vrow[x] = load_words<VEC>(P.V + (size_t)(r0 + r) * W + w0);
      else
#pragma unroll
        for (int i = 0; i < (int)VEC; i++) vrow[x].x[i] = 0xffffffffu;
    }
    if (!tile && sub == 0) {
      // A piece of a long row: the bits the row's other pieces have already
      // gathered this level count as reached, so once the level has
      // reached the row from every searching source its remaining pieces
      // gather nothing (they still arrive, so the last one writes the row).
      const uint32_t row_lo = __ldg(P.off + r0);
      const uint32_t first = (unit.c & 0x7fffffffu) - (unit.b - row_lo) / kPieceEntries;
      const uint32_t* na = P.nacc + (size_t)first * W + w0;
#pragma unroll
      for (int i = 0; i < (int)VEC; i++) vrow[0].x[i] |= __ldcg(na + i);
    }
    uint32_t needy = 0;
#pragma unroll
    for (uint32_t x = 0; x < VR; x++) {
      if (x * G >= R) break;
      bool nd = false;
#pragma unroll
      for (int i = 0; i < (int)VEC; i++) nd |= (~vrow[x].x[i] & a.x[i]) != 0;
      const uint32_t gb = __ballot_sync(0xffffffffu, nd);
      if constexpr (LPR == 1) {
        needy |= gb << (x * G);
      } else {
#pragma unroll
        for (uint32_t g = 0; g < G; g++)
          if ((gb >> (g * LPR)) & GM) needy |= 1u << (x * G + g);
      }
    }
    needy &= R == 32 ? 0xffffffffu : ((1u << R) - 1);
    uint32_t base, count;
    if (tile) {
      uint32_t lo = 0, hi = 0;
      if (lane < R) {
        lo = __ldg(P.off + r0 + lane);
        hi = __ldg(P.off + r0 + lane + 1);
      }
      base = unit.d;
      count = unit.c;
      if (needy)
        for (uint32_t k = lo - base; k < hi - base; k++) sm.rowof[k] = (uint8_t)lane;
      // The accumulators start as the rows' visited words (the registers
      // holding them are then free for the gathers).
#pragma unroll
      for (uint32_t x = 0; x < VR; x++) {
        const uint32_t r = x * G + sub;
        if (r < R) store_words<VEC>(&sm.acc[r * W + w0], vrow[x]);
      }
    } else {
      base = unit.b;
      count = unit.d - unit.b;
    }
    __syncwarp();
    // The hits: entries whose source row is in the frontier, in needy rows.
    uint32_t H = 0;
    if (needy) {
      uint32_t jv[Q];
#pragma unroll
      for (int qq = 0; qq < Q; qq++) {
        const uint32_t k = lane + 32 * qq;
        jv[qq] = k < count ? __ldcs(P.tgt + base + k) : 0u;
      }
      bool fb[Q];
#pragma unroll
      for (int qq = 0; qq < Q; qq++) fb[qq] = (lane + 32 * qq) < count && nbit(P.fbits, jv[qq]);
#pragma unroll
      for (int qq = 0; qq < Q; qq++) {
        const uint32_t k = lane + 32 * qq;
        const uint32_t row = (tile && fb[qq]) ? sm.rowof[k] : 0u;
        const bool hit = fb[qq] && ((needy >> row) & 1);
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
          const uint32_t pos = H + __popc(m & ((1u << lane) - 1));
          sm.hitj[pos] = jv[qq];
          sm.hitr[pos] = (uint8_t)row;
        }
        H += __popc(m);
      }
    }
    __syncwarp();
    // Gather the hit rows.  Lane group g takes the contiguous run of hits
    // [g·H/G, (g+1)·H/G) in order, U frontier rows in flight; the hits of
    // one row are consecutive, so they are OR-ed in registers and the row's
    // words are added to its accumulator once, when the row changes (atomic
    // ORs, as a row may straddle two groups' runs).  A piece is one row:
    // its words gather in `racc`.
    V4 racc = {};
    if (H) {
      const uint32_t per = (H + G - 1) / G;
      const uint32_t h_lo = min(H, sub * per), h_hi = min(H, sub * per + per);
      uint32_t cur = h_lo < h_hi ? sm.hitr[h_lo] : 0u;
      V4 run = {};
      for (uint32_t h0 = h_lo; h0 < h_hi; h0 += U) {
        V4 val[U];
#pragma unroll
        for (int x = 0; x < U; x++) {
          const uint32_t h = h0 + x;
          if (h < h_hi) {
            val[x] = ldg_words<VEC>(P.Fcur + (size_t)sm.hitj[h] * W + w0);
          } else {
#pragma unroll
            for (int i = 0; i < (int)VEC; i++) val[x].x[i] = 0;
          }
        }
#pragma unroll
        for (int x = 0; x < U; x++) {
          // The hit's row, read again here rather than held through the loads.
          const uint32_t rrx = h0 + x < h_hi ? sm.hitr[h0 + x] : cur;
          if (rrx != cur) {
#pragma unroll
            for (int i = 0; i < (int)VEC; i++)
              if (run.x[i] & a.x[i]) atomicOr(&sm.acc[cur * W + w0 + i], run.x[i] & a.x[i]);
#pragma unroll
            for (int i = 0; i < (int)VEC; i++) run.x[i] = 0;
            cur = rrx;
          }
#pragma unroll
          for (int i = 0; i < (int)VEC; i++) run.x[i] |= val[x].x[i];
        }
      }
      if (tile) {
#pragma unroll
        for (int i = 0; i < (int)VEC; i++)
          if (run.x[i] & a.x[i]) atomicOr(&sm.acc[cur * W + w0 + i], run.x[i] & a.x[i]);
      } else {
#pragma unroll
        for (int i = 0; i < (int)VEC; i++) racc.x[i] = run.x[i] & a.x[i];
      }
    }
    __syncwarp();
    if (tile) {
#pragma unroll
      for (uint32_t x = 0; x < VR; x++) {
        if (x * G >= R) break;
        const uint32_t r = x * G + sub;
        V4 fresh = {};
        if (r < R && ((needy >> r) & 1)) {
          // acc = V | gathered: the new bits are those V lacks.
          const V4 got = load_words<VEC>(&sm.acc[r * W + w0]);
          const V4 v = load_words<VEC>(P.V + (size_t)(r0 + r) * W + w0);
#pragma unroll
          for (int i = 0; i < (int)VEC; i++) fresh.x[i] = got.x[i] & ~v.x[i];
          if (any_words(fresh)) store_words<VEC>(P.V + (size_t)(r0 + r) * W + w0, got);
        }
        // Only rows with fresh bits are written (and marked so).
        const bool written = __ballot_sync(0xffffffffu, any_words(fresh)) & gmask;
        if (written) {
          store_words<VEC>(P.Fnext + (size_t)(r0 + r) * W + w0, fresh);
          if (q == 0) atomicOr(P.wbits_next + ((r0 + r) >> 5), 1u << ((r0 + r) & 31));
        }
        bool ex = false;
        const V4 a_next = load_words<VEC>(a_next_p);
#pragma unroll
        for (int i = 0; i < (int)VEC; i++) {
          live.x[i] |= fresh.x[i];
          ex |= (fresh.x[i] & a_next.x[i]) != 0;
        }
        const bool expands = __ballot_sync(0xffffffffu, ex) & gmask;
        if (r < R && expands && q == 0) {
          atomicOr(P.fbits_next + ((r0 + r) >> 5), 1u << ((r0 + r) & 31));
          admitted++;
          fed += __ldg(P.foff + r0 + r + 1) - __ldg(P.foff + r0 + r);
        }
      }
      __syncwarp();
    } else {
      // OR the lane groups' words together, then into the row's accumulator.
#pragma unroll
      for (uint32_t o = LPR; o < 32; o <<= 1)
#pragma unroll
        for (int i = 0; i < (int)VEC; i++) racc.x[i] |= __shfl_xor_sync(0xffffffffu, racc.x[i], o);
      const uint32_t row = unit.a, slot = unit.c & 0x7fffffffu;
      const uint32_t row_lo = __ldg(P.off + row);
      const uint32_t deg = __ldg(P.off + row + 1) - row_lo;
      const uint32_t pieces = (deg + kPieceEntries - 1) / kPieceEntries;
      const uint32_t first = slot - (unit.b - row_lo) / kPieceEntries;
      uint32_t* nacc = P.nacc + (size_t)first * W + w0;
      if (sub == 0)
#pragma unroll
        for (int i = 0; i < (int)VEC; i++)
          if (racc.x[i]) atomicOr(nacc + i, racc.x[i]);
      __threadfence();
      __syncwarp();
      uint32_t arrived = 0;
      if (lane == 0) arrived = atomicAdd(P.counters + first, 1u);
      arrived = __shfl_sync(0xffffffffu, arrived, 0);
      if (arrived == pieces - 1) {
        __threadfence();
        V4 fresh = {};
        if (sub == 0) {
          const V4 v = load_words<VEC>(P.V + (size_t)row * W + w0);
#pragma unroll
          for (int i = 0; i < (int)VEC; i++) {
            const uint32_t tot = __ldcg(nacc + i);
            fresh.x[i] = tot & ~v.x[i] & a.x[i];
          }
          store_words<VEC>(nacc, V4{});
          if (any_words(fresh)) {
            V4 nv;
#pragma unroll
            for (int i = 0; i < (int)VEC; i++) nv.x[i] = v.x[i] | fresh.x[i];
            store_words<VEC>(P.V + (size_t)row * W + w0, nv);
          }
        }
        if (__ballot_sync(0xffffffffu, any_words(fresh))) {
          if (sub == 0) store_words<VEC>(P.Fnext + (size_t)row * W + w0, fresh);
          if (lane == 0) atomicOr(P.wbits_next + (row >> 5), 1u << (row & 31));
        }
        bool ex = false;
        const V4 a_next = load_words<VEC>(a_next_p);
#pragma unroll
        for (int i = 0; i < (int)VEC; i++) {
          live.x[i] |= fresh.x[i];
          ex |= (fresh.x[i] & a_next.x[i]) != 0;
        }
        const bool expands = __ballot_sync(0xffffffffu, sub == 0 && ex) != 0;
        if (lane == 0) {
          P.counters[first] = 0;
          if (expands) {
            atomicOr(P.fbits_next + (row >> 5), 1u << (row & 31));
            admitted++;
            fed += __ldg(P.foff + row + 1) - __ldg(P.foff + row);
          }
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    admitted += __shfl_down_sync(0xffffffffu, admitted, o);
    fed += __shfl_down_sync(0xffffffffu, fed, o);
  }
  if (lane == 0 && admitted) {
    atomicAdd(P.counts + P.L + 1, admitted);
    atomicAdd(P.fedges + P.L + 1, fed);
  }
#pragma unroll
  for (uint32_t o = LPR; o < 32; o <<= 1)
#pragma unroll
    for (int i = 0; i < (int)VEC; i++) live.x[i] |= __shfl_xor_sync(0xffffffffu, live.x[i], o);
  if (sub == 0)
#pragma unroll
    for (int i = 0; i < (int)VEC; i++)
      if (live.x[i]) atomicOr(P.alive + (P.L + 1) * W + w0 + i, live.x[i]);
}

// Push, step 1: the frontier rows' words (masked to the live sources) are
// OR-ed into the accumulators of their out-neighbours, walking the forward
// CSR's schedule (a long row's pieces spread over warps); the neighbours
// are marked touched.  Lane group g of a warp takes entries g, g+G, ... of a
// row.
template <int W>
__global__ void __launch_bounds__(256) msbfs_push_kernel(MsLevel P) {
  if (!level_runs(P) || !level_pushes(P)) return;
  constexpr uint32_t G = 32 / W;
  const unsigned lane = threadIdx.x & 31;
  const unsigned sub = lane / W, w = lane % W;
  const uint32_t a = P.masks[P.L * W + w] & P.alive[P.L * W + w];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < P.funit_count; u += warps) {
    const Unit unit = P.funits[u];
    const bool tile = (unit.c >> 31) == 0;
    const uint32_t r0 = unit.a;
    const uint32_t R = tile ? unit.b - unit.a : 1;
    const bool in_frontier = lane < R && nbit(P.fbits, r0 + lane);
    uint32_t rows = __ballot_sync(0xffffffffu, in_frontier);
    while (rows) {
      const uint32_t r = __ffs(rows) - 1;
      rows &= rows - 1;
      const uint32_t j = r0 + r;
      const uint32_t val = P.Fcur[(size_t)j * W + w] & a;
      if (!__ballot_sync(0xffffffffu, val != 0)) continue;
      const uint32_t lo = tile ? __ldg(P.foff + j) : unit.b;
      const uint32_t hi = tile ? __ldg(P.foff + j + 1) : unit.d;
      for (uint32_t e = lo + sub; e < hi; e += G) {
        const uint32_t i = __ldg(P.ftgt + e);
        if (val) atomicOr(P.acc + (size_t)i * W + w, val);
        if (w == 0 && !nbit(P.touched, i)) atomicOr(P.touched + (i >> 5), 1u << (i & 31));
      }
    }
  }
}

// Push, step 2: each touched row settles its accumulator as a pulled row
// does (fresh = acc & ~V), clears the accumulator and its touched bit.
template <int W>
__global__ void __launch_bounds__(256) msbfs_settle_kernel(MsLevel P) {
  if (!level_runs(P) || !level_pushes(P)) return;
  constexpr uint32_t G = 32 / W;
  const unsigned lane = threadIdx.x & 31;
  const unsigned sub = lane / W, w = lane % W;
  const unsigned gmask = (W == 32) ? 0xffffffffu : (((1u << W) - 1) << (sub * W));
  const uint32_t a_next = P.masks[(P.L + 1) * W + w];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t words = (P.n + 31) / 32;
  uint32_t admitted = 0;
  unsigned long long fed = 0;
  uint32_t live = 0;
  for (uint32_t t = warp; t < words; t += warps) {
    uint32_t bits = P.touched[t];
    if (!bits) continue;
    __syncwarp();
    if (lane == 0) P.touched[t] = 0;
    while (bits) {
      // Group g takes the g-th lowest touched row left.
      uint32_t mine = bits;
      for (uint32_t q = 0; q < sub; q++) mine &= mine - 1;
      for (uint32_t q = 0; q < G; q++) bits &= bits - 1;
      uint32_t fresh = 0;
      uint32_t i = 0;
      if (mine) {
        i = 32 * t + (__ffs(mine) - 1);
        uint32_t* ap = P.acc + (size_t)i * W + w;
        const uint32_t got = *ap;
        if (got) *ap = 0;
        const uint32_t v = P.V[(size_t)i * W + w];
        fresh = got & ~v;
        if (fresh) P.V[(size_t)i * W + w] = v | fresh;
      }
      const bool written = __ballot_sync(0xffffffffu, fresh != 0) & gmask;
      if (mine && written) {
        P.Fnext[(size_t)i * W + w] = fresh;
        if (w == 0) atomicOr(P.wbits_next + (i >> 5), 1u << (i & 31));
      }
      live |= fresh;
      const bool expands = __ballot_sync(0xffffffffu, (fresh & a_next) != 0) & gmask;
      if (mine && expands && w == 0) {
        atomicOr(P.fbits_next + (i >> 5), 1u << (i & 31));
        admitted++;
        fed += __ldg(P.foff + i + 1) - __ldg(P.foff + i);
      }
    }
  }
  level_totals<W>(P, admitted, fed, live);
}

// Depths from the kept frontiers, source-major, and each source's
// edges_traversed: Σ out-degree over the nodes it reached at a depth below
// its cap.  A block of 512 threads takes 64 nodes at a time, all sources of
// the pass, so that each source's bytes of the tile are one 64-byte run:
// 32-byte runs spread over a thousand rows 2^22 bytes apart reached under
// half the write bandwidth that 64-byte runs do.
// Phase 1: a thread per (node, word) — the lanes of a warp cover whole node
// rows, so each level's row is read coalesced (only rows marked written,
// every node's first four levels in flight before any is folded).  A
// ballot over the tile's written-row words, a level per lane, gives the
// node its written levels; a node no source reached stores 255s at once.
// Otherwise the node's frontier words fold into NB bit planes of the depth
// (plane b: the sources that reached it at a level with bit b set) and the
// unreached set, and an 8×8 bit-matrix transpose turns 8 planes × 8 sources
// into 8 depth bytes (unreached sources have every plane set: 255).  The 32
// bytes go to a node-major shared tile as two 16-byte stores; 16-byte group
// h of node row j sits at h ^ (2·(j/16)), which keeps phase 2's reads free
// of bank conflicts.
// Phase 2: a thread per (four sources, sixteen nodes) reads sixteen words of
// the tile, transposes the bytes of each four so a word is one source's
// four nodes, and stores each source's sixteen bytes; four lanes cover a
// source's 64 nodes in one 64-byte run.  The out-degrees of the nodes whose
// depth is below the source's cap (bytes compared four at a time, weighted
// by dp4a) are summed over the four lanes by shuffles into the source's
// shared sum; the sums go to the global counts once per block.

// Rows a0..a3 of a 4×4 byte matrix become its columns: afterwards a_t
// holds [a0.t, a1.t, a2.t, a3.t] of the inputs.
__device__ inline void byte_transpose4(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3) {
  const uint32_t p = __byte_perm(a0, a1, 0x5140), q = __byte_perm(a2, a3, 0x5140);
  const uint32_t r = __byte_perm(a0, a1, 0x7362), s = __byte_perm(a2, a3, 0x7362);
  a0 = __byte_perm(p, q, 0x5410);
  a1 = __byte_perm(p, q, 0x7632);
  a2 = __byte_perm(r, s, 0x5410);
  a3 = __byte_perm(r, s, 0x7632);
}

// The 8×8 bit matrix held as eight bytes (lo: bytes 0-3, hi: bytes 4-7;
// element (r, c) is bit c of byte r) transposed: three rounds of swapping
// the off-diagonal 1×1, 2×2 and 4×4 blocks.
__device__ inline void bit_transpose8(uint32_t& lo, uint32_t& hi) {
  uint32_t t;
  t = (lo ^ (lo >> 7)) & 0x00AA00AAu;
  lo ^= t ^ (t << 7);
  t = (hi ^ (hi >> 7)) & 0x00AA00AAu;
  hi ^= t ^ (t << 7);
  t = (lo ^ (lo >> 14)) & 0x0000CCCCu;
  lo ^= t ^ (t << 14);
  t = (hi ^ (hi >> 14)) & 0x0000CCCCu;
  hi ^= t ^ (t << 14);
  t = (lo ^ (hi << 4)) & 0xF0F0F0F0u;
  lo ^= t;
  hi ^= t >> 4;
}

// Per byte, 1 where a < b (unsigned), else 0.  The low seven bits are
// compared by a subtraction that cannot borrow across bytes; the top bits
// decide where they differ.
__device__ inline uint32_t bytes_below(uint32_t a, uint32_t b) {
  const uint32_t x = (a | 0x80808080u) - (b & 0x7F7F7F7Fu);
  return (((~a & b) | (~(a ^ b) & ~x)) & 0x80808080u) >> 7;
}

// Item x's node's written levels: bit L set where level L's words of the
// tile (lane L holds the words of the tile's 64 nodes) have the node's bit.
// One ballot per node the warp covers (32 / W of them); every lane of the
// warp must call it.
template <int W>
__device__ inline uint32_t written_levels(const uint32_t (&wl)[2], uint32_t x, uint32_t lane,
                                          bool valid) {
  constexpr uint32_t NPW = 32 / W;
  const uint32_t jbase = (x - lane) / W;  // the warp's first node
  uint32_t lm = 0;
#pragma unroll
  for (uint32_t jj = 0; jj < NPW; jj++) {
    const uint32_t node = jbase + jj;
    const uint32_t word = node < 32 ? wl[0] : wl[1];
    const uint32_t bal = __ballot_sync(0xffffffffu, (word >> (node & 31)) & 1u);
    if (lane / W == jj) lm = bal;
  }
  return valid ? lm : 0u;
}

// A depth block is two teams of 512 threads: the producers fold a tile's
// levels into depth bytes (phase 1) while the consumers store the tile
// before it (phase 2), the tile double-buffered in shared memory and handed
// over through named barriers, so the stores of one tile run beside the
// folds of the next instead of after them.
constexpr uint32_t kDepthThreads = 512;    // producers
constexpr uint32_t kDepthConsumers = 512;
constexpr uint32_t kDepthBlock = kDepthThreads + kDepthConsumers;
constexpr uint32_t kDepthNodes = 64;

// Named barriers of the depth block: 1 + b (tile buffer b full), 3 + b
// (buffer b free), 5 (the consumers alone).
// Every warp of a team reaches each of them converged; each team's
// arrivals are matched one for one by the other team's waits, so at most
// one generation of a barrier is ever open.
__device__ inline void depth_bar_sync(uint32_t id, uint32_t count) {
  __syncwarp();
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ inline void depth_bar_arrive(uint32_t id, uint32_t count) {
  __syncwarp();
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// The depth kernel's dynamic shared memory: the tile, the caps, the sums
// and the tile's degrees.
template <int W> constexpr size_t depth_smem_bytes() {
  return 2 * (size_t)kDepthNodes * 8 * W * 4 + 32 * W * 4 + 32 * W * 8 + 2 * kDepthNodes * 4 +
         2 * (kDepthNodes / 4) * 16;
}

template <int W, int NB>
__global__ void __launch_bounds__(kDepthBlock, 1)
    msbfs_depth_kernel(uint32_t n, uint32_t k, uint32_t levels, const uint32_t* F, uint64_t fstride,
                       const uint32_t* wbits, uint32_t bitmap_words, const uint32_t* caps,
                       const uint32_t* off, const uint32_t* counts, uint8_t* depth_out,
                       unsigned long long* edges) {
  constexpr uint32_t S = 32 * W;            // sources in the pass (k <= S)
  constexpr uint32_t TN = kDepthNodes;      // nodes of a tile
  constexpr uint32_t Q = 8 * W;             // four-source words in a node row of the tile
  constexpr uint32_t IT = (TN * W + kDepthThreads - 1) / kDepthThreads;  // phase-1 items a thread takes
  constexpr uint32_t LC = NB == 5 ? 1 : 8;  // 32-level chunks of the written levels
  extern __shared__ __align__(16) unsigned char depth_smem[];
  uint32_t* tiles2 = reinterpret_cast<uint32_t*>(depth_smem);                  // [2][TN][Q]
  uint32_t* cap4s = tiles2 + 2 * TN * Q;                                        // [S]
  unsigned long long* esum = reinterpret_cast<unsigned long long*>(cap4s + S);  // [S]
  uint32_t* degs2 = reinterpret_cast<uint32_t*>(esum + S);                      // [2][TN]
  // Per node quad: the degrees' low and high bytes as byte planes (for
  // dp4a) and whether a degree is 2^16 or more (then the plain sum).
  uint4* dplanes2 = reinterpret_cast<uint4*>(degs2 + 2 * TN);                   // [2][TN / 4]
  const bool producer = threadIdx.x < kDepthThreads;
  const uint32_t lane = threadIdx.x & 31;
  // The snapshots written: F_L exists for L < used (F_L is written only if
  // level L-1 had a frontier to expand).
  uint32_t used = 1;
  while (used < levels && counts[used - 1] != 0) used++;
  for (uint32_t x = threadIdx.x; x < S; x += blockDim.x) {
    esum[x] = 0;
    // Depth bytes below the cap count as expanded; 255 marks "not reached".
    // With five planes depths are at most 31, so a cap above 127 compares
    // as 127 (the one-subtraction compare of phase 2 needs caps <= 127).
    cap4s[x] = (x < k ? min(caps[x], NB == 5 ? 127u : 255u) : 0u) * 0x01010101u;
  }
  // Word and 16-byte stores need the rows (and the caller's buffer) to
  // start on such boundaries; otherwise bytes are stored one at a time.
  const uintptr_t base = reinterpret_cast<uintptr_t>(depth_out);
  const bool aligned = (n & 3u) == 0 && (base & 3u) == 0;
  const bool aligned16 = (n & 15u) == 0 && (base & 15u) == 0;
  const uint32_t tiles = (n + TN - 1) / TN;
  __syncthreads();  // the caps and sums, before the teams part
  for (uint32_t t = blockIdx.x, li = 0; t < tiles; t += gridDim.x, li++) {
    const uint32_t i0 = t * TN;
    const uint32_t buf = li & 1;
    uint32_t* tile = tiles2 + buf * TN * Q;     // [TN][Q]
    uint32_t* degs = degs2 + buf * TN;          // [TN]
    uint4* dplanes = dplanes2 + buf * (TN / 4);  // [TN / 4]
    if (producer) {
    // The consumers are done with this buffer's tile before last.
    if (li >= 2) depth_bar_sync(3 + buf, kDepthBlock);
    // Lane L holds level 32c + L's written-row words of the tile's nodes.
    uint32_t wl[LC][2];
#pragma unroll
    for (uint32_t c = 0; c < LC; c++) {
      const uint32_t L = 32 * c + lane;
#pragma unroll
      for (uint32_t b = 0; b < 2; b++) {
        const uint32_t wi = 2 * t + b;
        wl[c][b] = L < used && wi < bitmap_words ? wbits[(size_t)L * bitmap_words + wi] : 0u;
      }
    }
    if (threadIdx.x < TN) {  // two whole warps
      const uint32_t i = i0 + threadIdx.x;
      const uint32_t dg = i < n ? __ldg(off + i + 1) - __ldg(off + i) : 0u;
      degs[threadIdx.x] = dg;
      // Lanes 4q .. 4q + 3 hold quad q's degrees: OR their bytes together.
      const uint32_t sh = 8 * (threadIdx.x & 3);
      uint32_t p0 = (dg & 0xffu) << sh, p1 = ((dg >> 8) & 0xffu) << sh;
      p0 |= __shfl_xor_sync(0xffffffffu, p0, 1);
      p1 |= __shfl_xor_sync(0xffffffffu, p1, 1);
      p0 |= __shfl_xor_sync(0xffffffffu, p0, 2);
      p1 |= __shfl_xor_sync(0xffffffffu, p1, 2);
      const uint32_t wq = __ballot_sync(0xffffffffu, (dg >> 16) != 0);
      if ((threadIdx.x & 3) == 0)
        dplanes[threadIdx.x >> 2] = make_uint4(p0, p1, (wq >> (threadIdx.x & 28)) & 0xfu, 0u);
    }
    // Phase 1a: every item's written levels 0..31 and the loads of its
    // first four, all in flight before any item is folded.
    uint32_t lm0[IT], fv[IT][4];
#pragma unroll
    for (uint32_t it = 0; it < IT; it++) {
      const uint32_t x = threadIdx.x + kDepthThreads * it;
      lm0[it] = 0;
#pragma unroll
      for (int u = 0; u < 4; u++) fv[it][u] = 0;
      if (x < TN * W) {
        const uint32_t j = x / W, w = x % W;
        lm0[it] = written_levels<W>(wl[0], x, lane, i0 + j < n);
        const uint32_t* row = F + (size_t)(i0 + j) * W + w;
        uint32_t m = lm0[it];
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (m) {
            fv[it][u] = __ldg(row + (size_t)(__ffs(m) - 1) * fstride);
            m &= m - 1;
          }
      }
    }
    // Phase 1b: fold each item's levels into planes and bytes.
#pragma unroll
    for (uint32_t it = 0; it < IT; it++) {
      const uint32_t x = threadIdx.x + kDepthThreads * it;
      if (x >= TN * W) break;
      const uint32_t j = x / W, w = x % W;
      uint32_t lm[LC];
      lm[0] = lm0[it];
      uint32_t any = lm[0];
#pragma unroll
      for (uint32_t c = 1; c < LC; c++) {
        lm[c] = written_levels<W>(wl[c], x, lane, i0 + j < n);
        any |= lm[c];
      }
      // The row's 16-byte group h sits at h ^ sw.
      const uint32_t sw = (2 * (j >> 4)) & (2 * W - 1);
      uint32_t* trow = tile + j * Q;
      uint4* grp0 = reinterpret_cast<uint4*>(trow + (((2 * w) ^ sw) << 2));
      uint4* grp1 = reinterpret_cast<uint4*>(trow + (((2 * w + 1) ^ sw) << 2));
      if (any == 0) {
        *grp0 = make_uint4(~0u, ~0u, ~0u, ~0u);
        *grp1 = make_uint4(~0u, ~0u, ~0u, ~0u);
        continue;
      }
      const uint32_t* row = F + (size_t)(i0 + j) * W + w;
      uint32_t P[NB];
#pragma unroll
      for (int b = 0; b < NB; b++) P[b] = 0;
      uint32_t reached = 0;
      {
        // The levels loaded in phase 1a (at most four).
        uint32_t m = lm[0];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if (!m) break;
          const uint32_t L = __ffs(m) - 1;
          m &= m - 1;
          const uint32_t f = fv[it][u];
          reached |= f;
#pragma unroll
          for (int b = 0; b < NB; b++)
            if ((L >> b) & 1u) P[b] |= f;
        }
        lm[0] = m;
      }
#pragma unroll
      for (uint32_t c = 0; c < LC; c++) {
        uint32_t m = lm[c];
        while (m) {
          uint32_t Ls[4], f[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            Ls[u] = 0;
            f[u] = 0;
            if (m) {
              Ls[u] = 32 * c + __ffs(m) - 1;
              m &= m - 1;
              f[u] = __ldg(row + (size_t)Ls[u] * fstride);
            }
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            reached |= f[u];
#pragma unroll
            for (int b = 0; b < NB; b++)
              if ((Ls[u] >> b) & 1u) P[b] |= f[u];
          }
        }
      }
      const uint32_t U = ~reached;
#pragma unroll
      for (int b = 0; b < NB; b++) P[b] |= U;
      // lo[g], hi[g]: byte b is plane b's byte g (planes NB..7 are U).
      uint32_t lo[4] = {P[0], P[1], P[2], P[3]}, hi[4];
      byte_transpose4(lo[0], lo[1], lo[2], lo[3]);
      if constexpr (NB == 5) {
#pragma unroll
        for (uint32_t g = 0; g < 4; g++)
          hi[g] = __byte_perm(P[4], U, g | (4 + g) << 4 | (4 + g) << 8 | (4 + g) << 12);
      } else {
        hi[0] = P[4];
        hi[1] = P[5];
        hi[2] = P[6];
        hi[3] = P[7];
        byte_transpose4(hi[0], hi[1], hi[2], hi[3]);
      }
#pragma unroll
      for (int g = 0; g < 4; g++) bit_transpose8(lo[g], hi[g]);
      // Sources 32w + 8g .. +3 are lo[g], +4 .. +7 hi[g]: the word's 16-byte
      // groups are 2w and 2w + 1.
      *grp0 = make_uint4(lo[0], hi[0], lo[1], hi[1]);
      *grp1 = make_uint4(lo[2], hi[2], lo[3], hi[3]);
    }
    depth_bar_arrive(1 + buf, kDepthBlock);
    } else {
    depth_bar_sync(1 + buf, kDepthBlock);
    // Phase 2: lanes 4h .. 4h + 3 of a warp take source quad g, lane p of
    // them nodes 16p .. 16p + 15 (node quads 4p .. 4p + 3).
    for (uint32_t y = threadIdx.x - kDepthThreads; y < Q * 4; y += kDepthConsumers) {
      const uint32_t g = y >> 2, p = y & 3;
      const uint4 c4 = *reinterpret_cast<const uint4*>(cap4s + 4 * g);
      const uint32_t cap[4] = {c4.x, c4.y, c4.z, c4.w};
      uint32_t o[4][4];  // [node quad][source]
      uint32_t part[4] = {0, 0, 0, 0};
#pragma unroll
      for (uint32_t h = 0; h < 4; h++) {
        const uint32_t q = 4 * p + h;
        const uint32_t col = (((g >> 2) ^ ((2 * p) & (2 * W - 1))) << 2) | (g & 3);
#pragma unroll
        for (uint32_t r = 0; r < 4; r++) o[h][r] = tile[(4 * q + r) * Q + col];
        // o[h][t]: source 4g + t at nodes 4q .. 4q + 3.
        byte_transpose4(o[h][0], o[h][1], o[h][2], o[h][3]);
        // The degrees' low two bytes as byte planes; a node of degree 2^16
        // or more takes the plain sum.
        const uint4 dp = dplanes[q];
        const bool wide = dp.z != 0;
        const uint32_t b0 = dp.x, b1 = dp.y;
#pragma unroll
        for (int t4 = 0; t4 < 4; t4++) {
          uint32_t lt;
          if constexpr (NB == 5) {
            // Depths are at most 31 or 255 and caps at most 127: (0x80 |
            // depth) - cap cannot borrow, and its bit 7 is set where
            // depth >= cap.
            lt = (~((o[h][t4] | 0x80808080u) - cap[t4]) & 0x80808080u) >> 7;
          } else {
            lt = bytes_below(o[h][t4], cap[t4]);
          }
          if (!wide)
            part[t4] += __dp4a(lt, b0, 0u) + (__dp4a(lt, b1, 0u) << 8);
          else {
            const uint4 d = *reinterpret_cast<const uint4*>(degs + 4 * q);
            part[t4] += (lt & 1u ? d.x : 0u) + ((lt >> 8) & 1u ? d.y : 0u) +
                        ((lt >> 16) & 1u ? d.z : 0u) + ((lt >> 24) & 1u ? d.w : 0u);
          }
        }
      }
      // Sum over the four lanes of the source quad: afterwards a lane holds
      // source 4g + 2·(lane bit 0) + (lane bit 1).
      const bool b0l = lane & 1u, b1l = lane & 2u;
      uint32_t v0 = b0l ? part[2] : part[0], v1 = b0l ? part[3] : part[1];
      v0 += __shfl_xor_sync(0xffffffffu, b0l ? part[0] : part[2], 1);
      v1 += __shfl_xor_sync(0xffffffffu, b0l ? part[1] : part[3], 1);
      uint32_t sum = b1l ? v1 : v0;
      sum += __shfl_xor_sync(0xffffffffu, b1l ? v0 : v1, 2);
      const uint32_t mine = 4 * g + 2 * (lane & 1u) + ((lane >> 1) & 1u);
      if (mine < k) esum[mine] += sum;
      const uint32_t node = i0 + 16 * p;
      const bool whole = aligned16 && node + 16 <= n;
      uint8_t* dst = depth_out + (size_t)(4 * g) * n + node;
#pragma unroll
      for (uint32_t t4 = 0; t4 < 4; t4++, dst += n) {
        if (4 * g + t4 >= k) break;
        if (whole) {
          *reinterpret_cast<uint4*>(dst) = make_uint4(o[0][t4], o[1][t4], o[2][t4], o[3][t4]);
        } else {
          for (uint32_t h = 0; h < 4; h++) {
            const uint32_t nq = node + 4 * h;
            if (aligned && nq + 4 <= n)
              *reinterpret_cast<uint32_t*>(dst + 4 * h) = o[h][t4];
            else
              for (uint32_t r = 0; r < 4 && nq + r < n; r++) dst[4 * h + r] = (uint8_t)(o[h][t4] >> (8 * r));
          }
        }
      }
    }
    depth_bar_arrive(3 + buf, kDepthBlock);
    }
  }
  if (producer) {
    // Match the consumers' frees of the last two tiles, then leave.
    const uint32_t mine = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0u;
    for (uint32_t li = mine >= 2 ? mine - 2 : 0u; li < mine; li++)
      depth_bar_sync(3 + (li & 1), kDepthBlock);
    return;
  }
  depth_bar_sync(5, kDepthConsumers);
  for (uint32_t x = threadIdx.x - kDepthThreads; x < k; x += kDepthConsumers)
    if (esum[x]) atomicAdd(edges + x, esum[x]);
}

// Depths are bytes with 255 for "not reached", so a pass runs at most
// kMaxLevels levels.  When a source's cap is deeper than that, the pass is
// cut short; if some source still had nodes to expand at the cut (rows
// admitted to the frontier of level kMaxLevels for a source whose cap is
// above it), the result would differ from wc_bfs, and the call is refused
// with WC_UNSUPPORTED (the adapter keeps the native search) instead of
// answering short.  Searches that end within kMaxLevels levels are served
// whatever their caps.
constexpr uint32_t kMaxLevels = 254;

__global__ void msbfs_truncated_kernel(const uint32_t* counts_at_cut, DeviceError* err) {
  if (threadIdx.x == 0 && *counts_at_cut != 0) raise(err, WC_UNSUPPORTED, kMaxLevels);
}

// Centrality passes (wc_centrality): no depths; after the levels, a flag
// if the last level reached any node (the pass must be run deeper), and
// otherwise each node's counts added to its totals.
__global__ void msbfs_cut_kernel(const uint32_t* wbits_last, uint32_t words, int* cut) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x)
    if (wbits_last[i]) *cut = 1;
}

// For each node u, the sources of the pass that first reach it at level L
// are the bits of its row of F_L (rows marked written; level 0 is the
// sources themselves).  They are counted per 64-source batch and the
// totals taken in the order of compute/centrality/closeness.rs's batched
// measures (mod.rs:15-20): batch by batch, then by distance — reached and
// the distance sum as integers, the harmonic sum as count / distance added
// one at a time.
template <int W>
__global__ void __launch_bounds__(256) msbfs_centrality_kernel(uint32_t n, uint32_t levels,
                                                               const uint32_t* F, uint64_t fstride,
                                                               const uint32_t* wbits,
                                                               uint32_t bitmap_words, CentArgs c) {
  static_assert(W % 2 == 0, "whole 64-source batches");
  if (*(volatile const int*)c.cut) return;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t word = u >> 5, bit = u & 31;
    unsigned long long reached = 0, dsum = 0;
    double h = 0.0;
    bool loaded = false;
    for (uint32_t b = 0; b < W / 2; b++) {
      for (uint32_t L0 = 1; L0 <= levels; L0 += 32) {
        uint32_t lm = 0;  // written levels L0 .. L0 + 31
        for (uint32_t j = 0; j < 32 && L0 + j <= levels; j++)
          lm |= ((wbits[(size_t)(L0 + j) * bitmap_words + word] >> bit) & 1u) << j;
        while (lm) {
          const uint32_t L = L0 + __ffs(lm) - 1;
          lm &= lm - 1;
          const uint2 w2 = __ldg(reinterpret_cast<const uint2*>(F + (size_t)L * fstride +
                                                                (size_t)u * W) + b);
          const uint32_t cnt = __popc(w2.x) + __popc(w2.y);
          if (cnt) {
            if (!loaded) {
              h = c.harm[u];
              loaded = true;
            }
            reached += cnt;
            dsum += (unsigned long long)cnt * L;
            h = h + (double)cnt / (double)L;
          }
        }
      }
    }
    if (loaded) {
      c.reached[u] += reached;
      c.dsum[u] += dsum;
      c.harm[u] = h;
    }
  }
}

// One pass of up to 32·W sources.
template <int W>
wc_status run_pass(Ctx& ctx, BatchBuffers& b, const uint64_t* sources_dev, const uint32_t* caps_dev,
                   uint32_t k, uint32_t levels, bool clipped, uint8_t* depth_dev,
                   unsigned long long* edges_dev, uint32_t blocks_per_sm, const CentArgs* cent) {
  wc_version* v = ctx.v;
  const uint32_t n = (uint32_t)v->n;
  const uint64_t row_words = (uint64_t)n * W;
  const uint64_t fstride = row_words;
  cudaStream_t st = ctx.stream;
  // Zero V, the bitmaps, the live sets and the counts, and the sources'
  // rows of F_0; only rows marked written are read from any F_L.
  WC_CUDA(cudaMemsetAsync(b.V->ptr, 0, row_words * 4, st), ctx.detail);
  const uint64_t bitmap_words = (n + 31) / 32;
  const uint64_t maps = (uint64_t)(levels + 2) * bitmap_words;
  WC_CUDA(cudaMemsetAsync(b.bits->ptr, 0, 2 * maps * 4, st), ctx.detail);
  WC_CUDA(cudaMemsetAsync(b.counts->ptr, 0, (levels + 2) * 16, st), ctx.detail);
  uint32_t* V = b.V->as<uint32_t>();
  uint32_t* F = b.F->as<uint32_t>();
  uint32_t* fbits = b.bits->as<uint32_t>();
  uint32_t* wbits = fbits + maps;
  uint32_t* masks = b.masks->as<uint32_t>();
  uint32_t* alive = masks + (levels + 2) * W;
  uint32_t* counts = b.counts->as<uint32_t>();
  unsigned long long* fedges =
      reinterpret_cast<unsigned long long*>(b.counts->as<unsigned char>() + (levels + 2) * 8);
  const uint32_t* foff = v->fwd.offsets.as<uint32_t>();
  WC_CUDA(cudaMemsetAsync(alive, 0, (uint64_t)(levels + 2) * W * 4, st), ctx.detail);
  note_launch(), msbfs_clear_kernel<W><<<(k + 255) / 256, 256, 0, st>>>(sources_dev, k, F);
  note_launch(), msbfs_seed_kernel<W><<<std::max<uint32_t>(1, (std::max(k, (levels + 1) * W) + 255) / 256), 256, 0,
                         st>>>(sources_dev, caps_dev, k, levels + 1, n, V, F, fbits, wbits, masks,
                               alive, counts, foff, fedges);
  const DevCsr& csc = v->rev;
  const size_t level_smem = 8 * sizeof(MsWarpSmem<W>);
  if (level_smem > 48 * 1024)
    WC_CUDA(cudaFuncSetAttribute(msbfs_level_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)level_smem), ctx.detail);
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(
      max_blocks((int)blocks_per_sm), (csc.schedule.count + 7) / 8));
  const DevCsr& fwd = v->fwd;
  const uint32_t push_grid = std::max<uint32_t>(1, std::min<uint32_t>(
      max_blocks(8), (fwd.schedule.count + 7) / 8));
  const uint32_t settle_grid = std::max<uint32_t>(1, std::min<uint32_t>(
      max_blocks(8), (uint32_t)((bitmap_words + 7) / 8)));
  // Each level queues its push (scatter, settle) and its pull; the kernels
  // that the level's frontier does not call for return at once.
  ctx.phase_begin("level");
  for (uint32_t L = 0; L < levels; L++) {
    MsLevel P{n, csc.offsets.as<uint32_t>(), csc.targets.as<uint32_t>(), csc.schedule.units.as<Unit>(),
              csc.schedule.count, csc.schedule.counters.as<uint32_t>(), b.nacc->as<uint32_t>(), V,
              F + L * fstride, F + (L + 1) * fstride, fbits + L * bitmap_words,
              fbits + (L + 1) * bitmap_words, wbits + (L + 1) * bitmap_words, masks, alive, L,
              counts, fedges, foff, fwd.targets.as<uint32_t>(), fwd.schedule.units.as<Unit>(),
              fwd.schedule.count, v->m, b.acc->as<uint32_t>(), b.touched->as<uint32_t>(),
              b.pulled ? b.pulled->as<uint32_t>() : nullptr,
              csc.schedule.row_masks.as<uint32_t>()};
    note_launch(), msbfs_cancel_kernel<<<1, 32, 0, st>>>(v->cancel_dev, counts + L);
    note_launch(), msbfs_push_kernel<W><<<push_grid, 256, 0, st>>>(P);
    note_launch(), msbfs_settle_kernel<W><<<settle_grid, 256, 0, st>>>(P);
    // The pull alone is timed too ("pull"), for its roofline.
    ctx.phase_begin("pull");
    note_launch(), msbfs_level_kernel<W><<<grid, 256, level_smem, st>>>(P);
    ctx.phase_end();
  }
  ctx.phase_end();
  if (clipped)
    note_launch(), msbfs_truncated_kernel<<<1, 32, 0, st>>>(counts + levels, v->error.as<DeviceError>());
  if (cent) {
    if constexpr (W % 2 == 0) {
      // Rows first reached at the last level (F_levels's written rows) may
      // have neighbours deeper still.
      note_launch(), msbfs_cut_kernel<<<max_blocks(2), 256, 0, st>>>(
          wbits + (uint64_t)levels * bitmap_words, (uint32_t)bitmap_words, cent->cut);
      if (!cent->keep_only)
        note_launch(), msbfs_centrality_kernel<W><<<max_blocks(4), 256, 0, st>>>(
            n, levels, F, fstride, wbits, (uint32_t)bitmap_words, *cent);
      return cuda_status(cudaGetLastError(), ctx.detail, "centrality pass");
    } else {
      return WC_INVALID_ARGUMENT;
    }
  }
  // Depths: persistent blocks of 64-node tiles (a producer and a consumer
  // team each), one block an SM.
  const uint32_t depth_grid = max_blocks(1);
  constexpr size_t depth_smem = depth_smem_bytes<W>();
  ctx.phase_begin("depth");
  // Depths fit five bit planes up to level 31.
  if (levels + 1 <= 32) {
    WC_CUDA(cudaFuncSetAttribute(msbfs_depth_kernel<W, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)depth_smem), ctx.detail);
    note_launch(), msbfs_depth_kernel<W, 5><<<depth_grid, kDepthBlock, depth_smem, st>>>(
        n, k, levels + 1, F, fstride, wbits, (uint32_t)bitmap_words, caps_dev,
        v->fwd.offsets.as<uint32_t>(), counts, depth_dev, edges_dev);
  } else {
    WC_CUDA(cudaFuncSetAttribute(msbfs_depth_kernel<W, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)depth_smem), ctx.detail);
    note_launch(), msbfs_depth_kernel<W, 8><<<depth_grid, kDepthBlock, depth_smem, st>>>(
        n, k, levels + 1, F, fstride, wbits, (uint32_t)bitmap_words, caps_dev,
        v->fwd.offsets.as<uint32_t>(), counts, depth_dev, edges_dev);
  }
  ctx.phase_end();
  return cuda_status(cudaGetLastError(), ctx.detail, "batched bfs pass");
}

wc_status BatchBuffers::reserve(Ctx& ctx, uint32_t words, uint32_t levels) {
  const uint64_t n = ctx.v->n;
  WC_TRY(ctx.scratch(POOL_BATCH_0, n * words * 4, &V));
  WC_TRY(ctx.scratch(POOL_BATCH_1, n * words * 4 * (uint64_t)(levels + 1), &F));
  // The frontier bitmaps and the written-row bitmaps, per level.
  WC_TRY(ctx.scratch(POOL_BATCH_2, ((n + 31) / 32) * 4 * (uint64_t)(levels + 2) * 2, &bits));
  // The level masks and the live sets, per level.
  WC_TRY(ctx.scratch(POOL_BATCH_3, (uint64_t)(levels + 2) * words * 4 * 2, &masks));
  // Per level: the admitted rows (u32) and their out-edges (u64).
  WC_TRY(ctx.scratch(POOL_BATCH_4, (uint64_t)(levels + 2) * 16, &counts));
  // The push accumulators and touched rows start zero and are left zero by
  // each level.
  {
    const uint64_t acc_bytes = n * words * 4, touched_bytes = ((n + 31) / 32) * 4;
    const bool fresh_acc = ctx.v->pool[POOL_MSBFS_ACC].bytes < acc_bytes;
    WC_TRY(ctx.scratch(POOL_MSBFS_ACC, acc_bytes, &acc));
    if (fresh_acc) WC_CUDA(cudaMemsetAsync(acc->ptr, 0, acc->bytes, ctx.stream), ctx.detail);
    const bool fresh_t = ctx.v->pool[POOL_MSBFS_TOUCHED].bytes < touched_bytes;
    WC_TRY(ctx.scratch(POOL_MSBFS_TOUCHED, touched_bytes, &touched));
    if (fresh_t) WC_CUDA(cudaMemsetAsync(touched->ptr, 0, touched->bytes, ctx.stream), ctx.detail);
  }
  // The long rows' accumulators start zero and are left zero by each level.
  const uint64_t nacc_bytes = (uint64_t)std::max<uint32_t>(ctx.v->rev.schedule.slots, 1) * words * 4;
  const bool fresh = ctx.v->pool[POOL_MSBFS_NACC].bytes < nacc_bytes;
  WC_TRY(ctx.scratch(POOL_MSBFS_NACC, nacc_bytes, &nacc));
  if (fresh) WC_CUDA(cudaMemsetAsync(nacc->ptr, 0, nacc->bytes, ctx.stream), ctx.detail);
  return WC_OK;
}

typedef wc_status (*PassFn)(Ctx&, BatchBuffers&, const uint64_t*, const uint32_t*, uint32_t,
                            uint32_t, bool, uint8_t*, unsigned long long*, uint32_t,
                            const CentArgs*);

static PassFn pass_for(uint32_t columns) {
  switch (columns) {
    case 32: return run_pass<1>;
    case 64: return run_pass<2>;
    case 128: return run_pass<4>;
    case 256: return run_pass<8>;
    case 512: return run_pass<16>;
    default: return run_pass<32>;
  }
}

static uint32_t round_columns(uint32_t k) {
  uint32_t c = 32;
  while (c < k && c < 1024) c <<= 1;
  return c;
}

wc_schedule default_bfs_schedule(uint32_t width) {
  return wc_schedule{round_columns(width), 1, 4, 0};
}

// The whole batch on the call's stream: passes of `columns` sources.
wc_status bfs_batched_run(Ctx& ctx, const wc_schedule& sched, const uint64_t* sources_dev,
                          const uint32_t* caps_dev, const uint32_t* caps_host, uint32_t width,
                          uint8_t* depth_dev, unsigned long long* edges_dev) {
  const uint32_t columns = std::max<uint32_t>(32, std::min<uint32_t>(1024, sched.columns_per_pass));
  BatchBuffers b;
  uint32_t max_levels = 0;
  for (uint32_t s = 0; s < width; s++) max_levels = std::max(max_levels, caps_host[s]);
  max_levels = std::min<uint32_t>(max_levels, kMaxLevels);
  WC_TRY(b.reserve(ctx, columns / 32, max_levels));
  if (ctx.timing) {
    WC_TRY(ctx.scratch(POOL_MSBFS_PULLED, 4, &b.pulled));
    WC_CUDA(cudaMemsetAsync(b.pulled->ptr, 0, 4, ctx.stream), ctx.detail);
  }
  WC_CUDA(cudaMemsetAsync(edges_dev, 0, width * 8, ctx.stream), ctx.detail);
  for (uint32_t s0 = 0; s0 < width; s0 += columns) {
    const uint32_t k = std::min(columns, width - s0);
    uint32_t levels = 0;
    for (uint32_t s = s0; s < s0 + k; s++) levels = std::max(levels, caps_host[s]);
    const bool clipped = levels > kMaxLevels;
    levels = std::min<uint32_t>(levels, kMaxLevels);
    const uint32_t bps = sched.blocks_per_sm ? sched.blocks_per_sm : 4;
    const std::string key = "bfs/" + std::to_string(columns) + "/" + std::to_string(k) + "/" +
                            std::to_string(levels) + "/" + std::to_string(bps) +
                            (clipped ? "/clipped" : "");
    WC_TRY(ctx.run_captured(key, [&] {
      return pass_for(columns)(ctx, b, sources_dev + s0, caps_dev + s0, k, levels, clipped,
                               depth_dev + (uint64_t)s0 * ctx.v->n, edges_dev + s0, bps, nullptr);
    }));
  }
  return WC_OK;
}

wc_status bfs_centrality_pass(Ctx& ctx, BatchBuffers& b, uint32_t columns,
                              const uint64_t* sources_dev, const uint32_t* caps_dev, uint32_t k,
                              uint32_t levels, uint32_t blocks_per_sm, const CentArgs& cent) {
  const std::string key = "cent/" + std::to_string(columns) + "/" + std::to_string(k) + "/" +
                          std::to_string(levels) + "/" + std::to_string(blocks_per_sm) +
                          (cent.keep_only ? "/keep" : "");
  return ctx.run_captured(key, [&] {
    return pass_for(columns)(ctx, b, sources_dev, caps_dev, k, levels, false, nullptr, nullptr,
                             blocks_per_sm, &cent);
  });
}

wc_status tune_minplus(Ctx& ctx, uint32_t width, wc_schedule* best);
wc_status tune_ppr(Ctx& ctx, uint32_t width, wc_schedule* best);

// Times `candidates` on a seeded sample batch of `width` sources (caps 16,
// the deepest the benchmark asks) and returns the fastest.
wc_status tune_bfs(Ctx& ctx, uint32_t width, wc_schedule* best) {
  wc_version* v = ctx.v;
  const uint32_t n = (uint32_t)v->n;
  std::vector<uint64_t> src(width);
  std::vector<uint32_t> caps(width, 16);
  uint64_t z = 0x7e57u;
  for (uint32_t s = 0; s < width; s++) {
    z = z * 6364136223846793005ull + 1442695040888963407ull;
    src[s] = (z >> 17) % n;
  }
  DevBuf *S, *C, *D, *E;
  WC_TRY(ctx.scratch(POOL_BATCH_5, width * 8, &S));
  WC_TRY(ctx.scratch(POOL_BATCH_6, width * 4, &C));
  WC_TRY(ctx.scratch(POOL_BATCH_7, (uint64_t)width * n, &D));
  WC_TRY(ctx.scratch(POOL_BATCH_9, width * 8, &E));
  WC_CUDA(cudaMemcpyAsync(S->ptr, src.data(), width * 8, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemcpyAsync(C->ptr, caps.data(), width * 4, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
  std::vector<wc_schedule> candidates;
  const uint32_t top = round_columns(width);
  for (uint32_t cols = top; cols >= 32 && cols * 4 >= top; cols >>= 1)
    for (uint32_t bps : {2u, 4u, 8u}) candidates.push_back(wc_schedule{cols, 1, bps, 0});
  cudaEvent_t a, b;
  WC_CUDA(cudaEventCreate(&a), ctx.detail);
  WC_CUDA(cudaEventCreate(&b), ctx.detail);
  float best_ms = 1e30f;
  for (const wc_schedule& c : candidates) {
    float ms = 0;
    for (int rep = 0; rep < 2; rep++) {  // the first run warms up
      WC_CUDA(cudaEventRecord(a, ctx.stream), ctx.detail);
      WC_TRY(bfs_batched_run(ctx, c, S->as<uint64_t>(), C->as<uint32_t>(), caps.data(), width,
                             D->as<uint8_t>(), E->as<unsigned long long>()));
      WC_CUDA(cudaEventRecord(b, ctx.stream), ctx.detail);
      WC_CUDA(cudaEventSynchronize(b), ctx.detail);
      WC_CUDA(cudaEventElapsedTime(&ms, a, b), ctx.detail);
    }
    if (ms < best_ms) {
      best_ms = ms;
      *best = c;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_schedule_set(wc_version* v, wc_batch_kind kind, uint32_t width,
                          const wc_schedule* schedule) {
  if (!v || !schedule || kind < WC_BATCH_BFS || kind > WC_BATCH_PPR) return WC_INVALID_ARGUMENT;
  const uint32_t c = schedule->columns_per_pass;
  if (c == 0 || c > 1024 || (c & (c - 1)) || (kind != WC_BATCH_BFS && (c > 32)) ||
      (kind == WC_BATCH_BFS && c < 32))
    return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  v->tuned[((uint64_t)kind << 32) | width] = *schedule;
  return WC_OK;
}

wc_status wc_autotune(wc_version* v, const wc_call* call, wc_batch_kind kind, uint32_t width,
                      wc_schedule* chosen) {
  if (!v || width == 0) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  WC_TRY(ctx.begin());
  wc_schedule best{};
  switch (kind) {
    case WC_BATCH_BFS: WC_TRY(tune_bfs(ctx, width, &best)); break;
    case WC_BATCH_MINPLUS: WC_TRY(tune_minplus(ctx, width, &best)); break;
    case WC_BATCH_PPR: WC_TRY(tune_ppr(ctx, width, &best)); break;
    default: return WC_INVALID_ARGUMENT;
  }
  WC_TRY(ctx.finish());
  v->tuned[((uint64_t)kind << 32) | width] = best;
  if (chosen) *chosen = best;
  return WC_OK;
}

wc_status wc_bfs_batched(wc_version* v, const wc_call* call, const uint64_t* sources,
                         const uint32_t* max_depths, uint32_t width, uint8_t* depth_out,
                         uint64_t* edges_traversed_out) {
  if (!v || (width && (!sources || !max_depths || !depth_out))) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  if (width == 0) return WC_OK;
  std::vector<uint64_t> src(width);
  std::vector<uint32_t> caps(width);
  WC_CUDA(cudaMemcpy(src.data(), sources, width * 8, cudaMemcpyDefault), ctx.detail);
  WC_CUDA(cudaMemcpy(caps.data(), max_depths, width * 4, cudaMemcpyDefault), ctx.detail);
  for (uint64_t s : src)
    if (s >= v->n) {
      if (ctx.detail) ctx.detail->node = s;
      return WC_NODE_OUTSIDE_ID_SPACE;
    }
  WC_TRY(ctx.begin());
  Operand S(POOL_BATCH_5), C(POOL_BATCH_6), D(POOL_BATCH_7), E(POOL_BATCH_8);
  WC_TRY(S.in(ctx, sources, width * 8));
  WC_TRY(C.in(ctx, max_depths, width * 4));
  WC_TRY(D.output(ctx, depth_out, (uint64_t)width * v->n));
  DevBuf* edges;
  WC_TRY(ctx.scratch(POOL_BATCH_9, (uint64_t)width * 8, &edges));
  auto key = ((uint64_t)WC_BATCH_BFS << 32) | width;
  wc_schedule sched = v->tuned.count(key) ? v->tuned[key] : default_bfs_schedule(width);
  WC_TRY(bfs_batched_run(ctx, sched, static_cast<const uint64_t*>(S.dev),
                         static_cast<const uint32_t*>(C.dev), caps.data(), width,
                         static_cast<uint8_t*>(D.dev), edges->as<unsigned long long>()));
  WC_TRY(D.out(ctx));
  if (edges_traversed_out)
    WC_CUDA(cudaMemcpyAsync(edges_traversed_out, edges->ptr, width * 8, cudaMemcpyDefault,
                            ctx.stream), ctx.detail);
  const wc_status st = ctx.finish();
  if (st == WC_OK && ctx.timing) {
    // The levels that pulled, for the pull's roofline (wc_version_timing).
    uint32_t pulled = 0;
    WC_CUDA(cudaMemcpy(&pulled, v->pool[POOL_MSBFS_PULLED].ptr, 4, cudaMemcpyDeviceToHost),
            ctx.detail);
    v->timings["pulled"] = {0.0, pulled};
  }
  if (st == WC_UNSUPPORTED)
    set_message(ctx.detail, "a search still expands at depth %u with a deeper cap; depths past %u "
                            "do not fit the byte output", kMaxLevels, kMaxLevels);
  return st;
}

}  // extern "C"
