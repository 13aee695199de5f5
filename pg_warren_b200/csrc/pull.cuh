// pull.cuh — the load-balanced pull kernel shared by SpMV, PageRank and the
// Lanczos operator: y_i = ⊕_{entries (i, j)} ⊗(w_ij, x_j) over a device CSR,
// walked by a precomputed row-split schedule.
//
// The reference folds each row sequentially in ascending column order, the
// first entry setting the sum (compute/product/kernel.rs:84-121).  Here a
// warp takes one unit of the schedule at a time:
//  - a tile of up to 32 consecutive rows holding at most 256 entries (its
//    first entry and entry count are in the descriptor): the tile's
//    targets, weights and row offsets arrive in the warp's shared-memory
//    ring by bulk copies issued a few units ahead, the warp gathers x
//    through the read-only path and stages the products, then each lane
//    folds one row sequentially from shared memory — the reference's order
//    exactly;
//  - a piece of up to 256 entries of a longer row: the warp stages its
//    products, each lane folds a contiguous run of 8, then the lanes combine
//    left to right; pieces of one row are combined in piece order by
//    whichever warp finishes the row's last piece.  Order-preserving
//    combines keep min/max (first on a tie), lor, any and the i64 checked
//    sum exactly what a sequential fold gives; only floating-point plus is
//    reassociated, and only in rows longer than 256 entries.
#pragma once

#include "bulk.cuh"
#include "product.h"
#include "semiring.cuh"

namespace wc {

constexpr int kPullThreads = 256;
constexpr int kPullWarps = kPullThreads / 32;

// One CSR orientation as the kernels read it.  W: double (f64 weights),
// int32_t (the integral copy) or void (unweighted: every weight 1).
// `hot`: over a locality-ordered CSC (nodes numbered by out-degree, largest
// first), the gathers of x_j with j < hot are kept in L1 and the others
// bypass it; 0 for a CSC in dense-id order (every gather as any other).
template <class W> struct CsrView {
  const uint32_t* off;
  const uint32_t* tgt;
  const W* w;
  const Unit* units;
  uint32_t unit_count;
  uint32_t* counters;
  void* carry;
  uint32_t hot = 0;
};
template <> struct CsrView<void> {
  const uint32_t* off;
  const uint32_t* tgt;
  const void* w;
  const Unit* units;
  uint32_t unit_count;
  uint32_t* counters;
  void* carry;
  uint32_t hot = 0;
};

// An entry's weight as stored (WT), loaded apart from its product so the
// loads of a tile can all be in flight at once.
template <class E, int S, class W> struct EntryOf;
template <class E, int S> struct EntryOf<E, S, double> {
  typedef double WT;
  __device__ static WT load(const CsrView<double>& A, uint32_t e) { return __ldcs(A.w + e); }
  __device__ static int32_t product(WT w, E xv, E* o) { return Entry<E, S, double>::product(w, xv, o); }
  __device__ static int32_t get(const CsrView<double>& A, uint32_t e, E xv, E* o) {
    return product(load(A, e), xv, o);
  }
};
template <class E, int S> struct EntryOf<E, S, int32_t> {
  typedef int32_t WT;
  __device__ static WT load(const CsrView<int32_t>& A, uint32_t e) { return __ldcs(A.w + e); }
  __device__ static int32_t product(WT w, E xv, E* o) {
    return Entry<E, S, int32_t>::product_int(w, xv, o);
  }
  __device__ static int32_t get(const CsrView<int32_t>& A, uint32_t e, E xv, E* o) {
    return product(load(A, e), xv, o);
  }
};
template <class E, int S> struct EntryOf<E, S, void> {
  typedef char WT;
  __device__ static WT load(const CsrView<void>&, uint32_t) { return 0; }
  __device__ static int32_t product(WT, E xv, E* o) { return Entry<E, S, void>::product(1.0, xv, o); }
  __device__ static int32_t get(const CsrView<void>&, uint32_t, E xv, E* o) {
    return product(0, xv, o);
  }
};

template <class E> __device__ inline E load_x(const E* x, uint32_t j) { return __ldg(x + j); }
template <> __device__ inline bool8 load_x<bool8>(const bool8* x, uint32_t j) {
  return *(x + j);
}

// A gather over a locality-ordered CSC: the few most gathered values (j <
// hot) are kept in L1, the rest are read past it so they do not evict those;
// in L2 every value is kept ahead of the streamed CSR (`keep`: an
// l2_evict_last_policy).  8-byte elements only; others take load_x.
template <class E>
__device__ inline E load_x_split(const E* x, uint32_t j, uint32_t hot, uint64_t keep) {
  if constexpr (sizeof(E) == 8) {
    unsigned long long b;
    if (j < hot)
      asm("ld.global.nc.L1::evict_last.L2::cache_hint.b64 %0, [%1], %2;"
          : "=l"(b) : "l"(x + j), "l"(keep));
    else
      asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b64 %0, [%1], %2;"
          : "=l"(b) : "l"(x + j), "l"(keep));
    E v;
    memcpy(&v, &b, 8);
    return v;
  } else {
    return load_x(x, j);
  }
}

// An accumulator with a presence flag: the first entry sets the sum.
template <class E, int ADD> struct alignas(16) Partial {
  Acc<E, ADD> acc;
  bool present;
};

// A load that bypasses L1, for values other blocks wrote during this launch.
template <class T> __device__ inline T load_cg(const T* p) {
  static_assert(sizeof(T) % 8 == 0, "8-byte multiples only");
  T r;
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(p);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&r);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 8); i++) d[i] = __ldcg(s + i);
  return r;
}

template <class E, int ADD>
__device__ inline Partial<E, ADD> join(Partial<E, ADD> a, Partial<E, ADD> b) {
  if (!a.present) return b;
  if (!b.present) return a;
  return Partial<E, ADD>{Acc<E, ADD>::combine(a.acc, b.acc), true};
}

template <class E, int ADD>
__device__ inline Partial<E, ADD> shfl_partial(const Partial<E, ADD>& p, unsigned off) {
  Partial<E, ADD> r;
  r.acc = p.acc.shfl_down(off);
  r.present = __shfl_down_sync(0xffffffffu, (int)p.present, off) != 0;
  return r;
}

// Counts a piece in: the release publishes this thread's carry store, the
// acquire (for the last to arrive) makes the other pieces' carries visible.
// Cheaper than a full fence before a relaxed atomic.
__device__ inline uint32_t arrive_acq_rel(uint32_t* counter) {
  uint32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
  return old;
}

// The combine of a long row's piece partials, in piece order, by the warp
// that brings the row's last piece: the warp's G = 32 / P lane groups (lane
// = g·P + c for column c) each fold a contiguous run of the pieces, then the
// groups combine left to right, so a row of many pieces costs about
// pieces / G dependent loads instead of `pieces`.  Group 0 holds the total.
template <class E, int ADD, int P>
__device__ inline Partial<E, ADD> combine_pieces(const Partial<E, ADD>* carry, uint32_t first,
                                                 uint32_t pieces, uint32_t c, uint32_t g) {
  constexpr uint32_t G = 32 / P;
  const uint32_t per = (pieces + G - 1) / G;
  const uint32_t p0 = min(pieces, g * per), p1 = min(pieces, g * per + per);
  Partial<E, ADD> mine{Acc<E, ADD>::of(E{}), false};
#pragma unroll 4
  for (uint32_t p = p0; p < p1; p++)
    mine = join(mine, load_cg(carry + (size_t)(first + p) * P + c));
  for (uint32_t o = P; o < 32; o <<= 1) {  // groups o/P apart: left to right
    Partial<E, ADD> other = shfl_partial(mine, o);
    if ((g & (2 * (o / P) - 1)) == 0) mine = join(mine, other);
  }
  return mine;
}

// ------------------------------------------------- the warp's staging ring
// Each warp keeps a ring of R buffers in shared memory.  Lane 0 fills a
// buffer with one unit's targets, weights and (for a tile) row offsets by
// bulk copies completed on the buffer's mbarrier, R units ahead of the unit
// the warp is folding, so the stream of the CSR is always in flight and a
// unit's critical path is one x gather.  Spans are widened to 16-byte
// boundaries (kSpan, kOffSpan); the CSR arrays carry 16 bytes of padding.

constexpr uint32_t kSpan = kTileEntries + 8;
constexpr uint32_t kOffSpan = kTileRows + 8;

template <class W> struct WSize { static constexpr int v = sizeof(W); };
template <> struct WSize<void> { static constexpr int v = 0; };
template <class W> struct alignas(16) WSpan { W v[kSpan]; };
template <> struct alignas(16) WSpan<void> {};

template <class E, class W> struct alignas(16) PullRing {
  static constexpr int R = WSize<W>::v == 0 ? 3 : 2;
  uint32_t tgt[R][kSpan];
  WSpan<W> w[R];
  uint32_t off[R][kOffSpan];
  Unit desc[R];
  E stage[kTileEntries];
  uint64_t bar[R];
};

template <class E, class W> constexpr size_t pull_smem_bytes() {
  return kPullWarps * sizeof(PullRing<E, W>);
}

// The first entry and entry count of a unit.
__device__ inline uint32_t unit_first(const Unit& d) { return (d.c >> 31) == 0 ? d.d : d.b; }
__device__ inline uint32_t unit_count(const Unit& d) { return (d.c >> 31) == 0 ? d.c : d.d - d.b; }

// Lane 0: fills buffer b with unit d, the CSR's spans streamed past L2's
// kept lines (`stream`: an l2_evict_first_policy).
template <class E, class W>
__device__ inline void issue_unit(const CsrView<W>& A, PullRing<E, W>* ring, int b, const Unit& d,
                                  uint64_t stream) {
  ring->desc[b] = d;
  const uint32_t e0 = unit_first(d), cnt = unit_count(d);
  const uint32_t ta = e0 & ~3u, tb = cnt ? (e0 + cnt + 3) & ~3u : ta;
  uint32_t bytes = (tb - ta) * 4;
  uint32_t wa = 0, wb = 0;
  if constexpr (WSize<W>::v == 8) {
    wa = e0 & ~1u;
    wb = cnt ? (e0 + cnt + 1) & ~1u : wa;
    bytes += (wb - wa) * 8;
  } else if constexpr (WSize<W>::v == 4) {
    wa = ta;
    wb = tb;
    bytes += (wb - wa) * 4;
  }
  const bool tile = (d.c >> 31) == 0;
  const uint32_t oa = d.a & ~3u, ob = (d.b + 1 + 3) & ~3u;
  if (tile) bytes += (ob - oa) * 4;
  mbar_arrive_expect(&ring->bar[b], bytes);
  if (tb > ta) bulk_load_hint(ring->tgt[b], A.tgt + ta, (tb - ta) * 4, &ring->bar[b], stream);
  if constexpr (WSize<W>::v != 0) {
    if (wb > wa)
      bulk_load_hint(ring->w[b].v, A.w + wa, (wb - wa) * WSize<W>::v, &ring->bar[b], stream);
  }
  if (tile) bulk_load_hint(ring->off[b], A.off + oa, (ob - oa) * 4, &ring->bar[b], stream);
}

// The weight of the k-th entry of the unit in buffer b.
template <class E, int S, class W>
__device__ inline typename EntryOf<E, S, W>::WT ring_weight(const PullRing<E, W>* ring, int b,
                                                            uint32_t e0, uint32_t k) {
  if constexpr (WSize<W>::v == 8) return ring->w[b].v[(e0 & 1u) + k];
  else if constexpr (WSize<W>::v == 4) return ring->w[b].v[(e0 & 3u) + k];
  else return 0;
}

// Stages the products of the unit in buffer b (count <= 256 entries) in the
// warp's stage: each lane gathers its (up to 8) x values at once, then forms
// the products.
template <class E, int S, class W, bool SPLIT>
__device__ inline void stage_products(const PullRing<E, W>* ring, int b, const E* __restrict__ x,
                                      uint32_t e0, uint32_t count, E* stage, DeviceError* err,
                                      uint32_t row, uint32_t hot, uint64_t keep) {
  const unsigned lane = threadIdx.x & 31;
  constexpr int Q = kTileEntries / 32;
  const uint32_t* tg = ring->tgt[b] + (e0 & 3u);
  E xv[Q];
  if constexpr (SPLIT) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const uint32_t k = lane + 32 * q;
      if (k < count) xv[q] = load_x_split(x, tg[k], hot, keep);
    }
  } else {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const uint32_t k = lane + 32 * q;
      if (k < count) xv[q] = load_x(x, tg[k]);
    }
  }
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const uint32_t k = lane + 32 * q;
    if (k < count) {
      E p;
      int32_t s = EntryOf<E, S, W>::product(ring_weight<E, S, W>(ring, b, e0, k), xv[q], &p);
      if (s) raise(err, s, row);
      stage[k] = p;
    }
  }
}

// Walks the schedule, a warp per unit, the units of a warp strided by the
// grid's warp count, through the warp's staging ring.  SPLIT: the CSC is in
// locality order and A.hot splits the gathers (load_x_split).  The epilogue's
// per-row operands (`epi.pre(row)`) are requested as a unit starts, so they
// arrive with its gathers.  `epi.row(row, present, value, pre)` is called
// exactly once per row, by one lane.  A ring wait that runs out (about 2 s)
// raises WC_DEVICE_TIMEOUT and ends the walk after the copies in flight.
template <class E, int S, class W, class Epi, bool SPLIT = false, bool DEFER = false>
__device__ inline void pull_units(const CsrView<W>& A, const E* __restrict__ x, Epi& epi,
                                  DeviceError* err, PullRing<E, W>* ring) {
  constexpr int R = PullRing<E, W>::R;
  constexpr int ADD = semiring_add(S);
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  Partial<E, ADD>* carry = static_cast<Partial<E, ADD>*>(A.carry);
  if (warp >= A.unit_count) return;

  if (lane == 0)
    for (int b = 0; b < R; b++) mbar_init(&ring->bar[b], 1);
  __syncwarp();
  const uint64_t stream = l2_evict_first_policy();
  uint64_t keep = 0;
  if constexpr (SPLIT) keep = l2_evict_last_policy();
  Unit ahead{0u, 0u, 0u, 0u};  // lane 0: the next unit to issue
  uint32_t pending = 0;        // buffers with a copy in flight (uniform)
  for (int b = 0; b < R; b++) {
    const uint32_t u = warp + b * warps;
    if (u < A.unit_count) {
      if (lane == 0) issue_unit(A, ring, b, A.units[u], stream);
      pending |= 1u << b;
    }
  }
  if (lane == 0 && warp + R * warps < A.unit_count) ahead = A.units[warp + R * warps];
  __syncwarp();

  uint32_t phase = 0;
  int b = 0;
  for (uint32_t u = warp; u < A.unit_count; u += warps) {
    const bool ok = mbar_wait(&ring->bar[b], (phase >> b) & 1u);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) raise(err, WC_DEVICE_TIMEOUT);
      for (int q = 0; q < R; q++)
        if (pending & (1u << q)) mbar_wait(&ring->bar[q], (phase >> q) & 1u);
      break;
    }
    phase ^= 1u << b;
    pending &= ~(1u << b);
    const Unit unit = ring->desc[b];
    if ((unit.c >> 31) == 0) {
      // A tile of rows [a, b) holding c entries from d: stage every
      // product, then one lane per row folds its run in column order.
      const uint32_t r0 = unit.a, rows = unit.b - unit.a, e0 = unit.d, count = unit.c;
      const uint32_t* soff = ring->off[b] + (r0 & 3u);
      uint32_t lo = 0, hi = 0;
      typename Epi::Pre pre{};
      if (lane < rows) {
        lo = soff[lane];
        hi = soff[lane + 1];
        pre = epi.pre(r0 + lane);
      }
      stage_products<E, S, W, SPLIT>(ring, b, x, e0, count, ring->stage, err, r0, A.hot, keep);
      __syncwarp();
      if (lane < rows) {
        E sum{};
        bool present = false;
        int32_t bad = 0;
        for (uint32_t k = lo - e0; k < hi - e0; k++) {
          E p = ring->stage[k];
          if (present) {
            int32_t s = Apply<E, ADD>::go(sum, p, &sum);
            if (s) bad = s;
          } else {
            sum = p;
            present = true;
          }
        }
        if (bad) raise(err, bad, r0 + lane);
        epi.row(r0 + lane, present, sum, pre);
      }
    } else {
      // A piece [b, d) (at most 256 entries) of row a: each lane folds a
      // contiguous run of 8, then the lanes combine left to right.
      const uint32_t row = unit.a, e0 = unit.b, e1 = unit.d;
      const uint32_t slot = unit.c & 0x7fffffffu;
      const uint32_t count = e1 - e0;
      stage_products<E, S, W, SPLIT>(ring, b, x, e0, count, ring->stage, err, row, A.hot, keep);
      __syncwarp();
      Partial<E, ADD> mine{Acc<E, ADD>::of(E{}), false};
      constexpr uint32_t per = kTileEntries / 32;
      for (uint32_t k = lane * per; k < min(count, lane * per + per); k++)
        mine = join(mine, Partial<E, ADD>{Acc<E, ADD>::of(ring->stage[k]), true});
      for (unsigned o = 1; o < 32; o <<= 1) {
        Partial<E, ADD> other = shfl_partial(mine, o);
        if ((lane & (2 * o - 1)) == 0) mine = join(mine, other);
      }
      if constexpr (DEFER) {
        // The piece's partial only: a later pass combines each long
        // row's pieces in order (it starts after every piece is stored).
        if (lane == 0) carry[slot] = mine;
      } else {
        const uint32_t row_lo = __ldg(A.off + row);
        const uint32_t deg = __ldg(A.off + row + 1) - row_lo;
        const uint32_t pieces = (deg + kPieceEntries - 1) / kPieceEntries;
        const uint32_t first = slot - (e0 - row_lo) / kPieceEntries;
        uint32_t arrived = 0;
        if (lane == 0) {
          carry[slot] = mine;
          arrived = arrive_acq_rel(A.counters + first);
        }
        arrived = __shfl_sync(0xffffffffu, arrived, 0);
        if (arrived == pieces - 1) {
          __threadfence();
          typename Epi::Pre pre{};
          if (lane == 0) pre = epi.pre(row);
          Partial<E, ADD> total = combine_pieces<E, ADD, 1>(carry, first, pieces, 0, lane);
          if (lane == 0) {
            A.counters[first] = 0;
            E v;
            int32_t s = total.acc.value(&v);
            if (s) raise(err, s, row);
            epi.row(row, true, v, pre);
          }
        }
      }
    }
    __syncwarp();
    // Refill this buffer with the unit R ahead.
    const uint32_t un = u + R * warps;
    if (un < A.unit_count) {
      if (lane == 0) {
        issue_unit(A, ring, b, ahead, stream);
        if (un + warps < A.unit_count) ahead = A.units[un + warps];
      }
      pending |= 1u << b;
    }
    __syncwarp();
    b = b + 1 == R ? 0 : b + 1;
  }
}

// ----------------------------------------------------------- the write
// compute/product/kernel.rs:200-240 (Write::row) and compute/mask.rs:34-44.

__device__ inline bool mask_selects(const WriteArgs& w, uint32_t row) {
  if (!w.mask) return true;
  bool set;
  switch (w.mask_dtype) {
    case WC_F32: { float v = static_cast<const float*>(w.mask)[row]; set = v != 0.0f || v != v; break; }
    case WC_F64: { double v = static_cast<const double*>(w.mask)[row]; set = v != 0.0 || v != v; break; }
    case WC_I64: set = static_cast<const int64_t*>(w.mask)[row] != 0; break;
    default: set = static_cast<const bool8*>(w.mask)[row] != 0; break;
  }
  return set != (w.complement != 0);
}

template <class E, int S> struct WriteEpi {
  WriteArgs w;
  E* y;
  DeviceError* err;
  // Whether the mask selects the row, and y's old value when it is
  // accumulated into.
  struct Pre {
    bool selected;
    E old;
  };
  __device__ Pre pre(uint32_t row) const {
    Pre p{mask_selects(w, row), E{}};
    if (w.accumulate >= 0 && p.selected) p.old = y[row];
    return p;
  }
  __device__ void row(uint32_t row, bool present, E t, const Pre& p) {
    const E identity = Identity<E>::of(semiring_add(S));
    if (!p.selected) {
      if (w.replace) y[row] = identity;
      return;
    }
    if (w.accumulate < 0) {
      y[row] = present ? t : identity;
    } else if (present) {
      E out;
      int32_t s = apply_rt<E>(w.accumulate, p.old, t, &out);
      if (s) raise(err, s, row);
      else y[row] = out;
    }
  }
};

}  // namespace wc
