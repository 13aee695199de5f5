// pull.cuh — the load-balanced pull kernel shared by SpMV, PageRank and the
// Lanczos operator: y_i = ⊕_{entries (i, j)} ⊗(w_ij, x_j) over a device CSR,
// walked by a precomputed row-split schedule.
//
// The reference folds each row sequentially in ascending column order, the
// first entry setting the sum (compute/product/kernel.rs:84-121).  Here a
// warp takes one unit of the schedule at a time:
//  - a tile of up to 32 consecutive rows holding at most 256 entries: the
//    warp stages the tile's products in shared memory with coalesced loads
//    (targets and weights streamed with an evict-first hint, x gathered
//    through the read-only path), then each lane folds one row sequentially
//    from shared memory — the reference's order exactly;
//  - a piece of up to 4096 entries of a longer row: the warp folds chunks of
//    256 staged products, each lane a contiguous run of 8, then combines the
//    lanes left to right; pieces of one row are combined in piece order by
//    whichever warp finishes the row's last piece.  Order-preserving
//    combines keep min/max (first on a tie), lor, any and the i64 checked
//    sum exactly what a sequential fold gives; only floating-point plus is
//    reassociated, and only in rows longer than 256 entries.
#pragma once

#include "product.h"
#include "semiring.cuh"

namespace wc {

constexpr int kPullThreads = 256;
constexpr int kPullWarps = kPullThreads / 32;

// One CSR orientation as the kernels read it.  W: double (f64 weights),
// int32_t (the integral copy) or void (unweighted: every weight 1).
template <class W> struct CsrView {
  const uint32_t* off;
  const uint32_t* tgt;
  const W* w;
  const Unit* units;
  uint32_t unit_count;
  uint32_t* counters;
  void* carry;
};
template <> struct CsrView<void> {
  const uint32_t* off;
  const uint32_t* tgt;
  const void* w;
  const Unit* units;
  uint32_t unit_count;
  uint32_t* counters;
  void* carry;
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

// Stages the products of entries [base, base + count) (count <= 256) in
// `stage`: every lane first issues its (up to 8) target loads, then its
// weight loads and x gathers, then forms the products, so each lane has
// eight independent loads in flight instead of a chain.
template <class E, int S, class W>
__device__ inline void stage_products(const CsrView<W>& A, const E* __restrict__ x, uint32_t base,
                                      uint32_t count, E* stage, DeviceError* err, uint32_t row) {
  const unsigned lane = threadIdx.x & 31;
  constexpr int Q = kTileEntries / 32;
  uint32_t j[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const uint32_t k = lane + 32 * q;
    j[q] = k < count ? __ldcs(A.tgt + base + k) : 0u;
  }
  E xv[Q];
  typename EntryOf<E, S, W>::WT wv[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const uint32_t k = lane + 32 * q;
    if (k < count) {
      xv[q] = load_x(x, j[q]);
      wv[q] = EntryOf<E, S, W>::load(A, base + k);
    }
  }
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const uint32_t k = lane + 32 * q;
    if (k < count) {
      E p;
      int32_t s = EntryOf<E, S, W>::product(wv[q], xv[q], &p);
      if (s) raise(err, s, row);
      stage[k] = p;
    }
  }
}

// Walks the schedule.  `epi.row(row, present, value)` is called exactly
// once per row, by one lane.  Products are staged in `stage`
// (kTileEntries elements per warp).
template <class E, int S, class W, class Epi>
__device__ inline void pull_units(const CsrView<W>& A, const E* __restrict__ x, Epi& epi,
                                  DeviceError* err, E* stage) {
  constexpr int ADD = semiring_add(S);
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  Partial<E, ADD>* carry = static_cast<Partial<E, ADD>*>(A.carry);

  for (uint32_t u = warp; u < A.unit_count; u += warps) {
    const Unit unit = A.units[u];
    if ((unit.c >> 31) == 0) {
      // A tile of rows [a, b): stage every product, then one lane per row.
      const uint32_t r0 = unit.a, rows = unit.b - unit.a;
      uint32_t lo = 0, hi = 0;
      if (lane < rows) {
        lo = __ldg(A.off + r0 + lane);
        hi = __ldg(A.off + r0 + lane + 1);
      }
      const uint32_t base = __shfl_sync(0xffffffffu, lo, 0);
      const uint32_t end = __shfl_sync(0xffffffffu, hi, rows - 1);
      stage_products<E, S, W>(A, x, base, end - base, stage, err, r0);
      __syncwarp();
      if (lane < rows) {
        E sum{};
        bool present = false;
        int32_t bad = 0;
        for (uint32_t k = lo - base; k < hi - base; k++) {
          E p = stage[k];
          if (present) {
            int32_t s = Apply<E, ADD>::go(sum, p, &sum);
            if (s) bad = s;
          } else {
            sum = p;
            present = true;
          }
        }
        if (bad) raise(err, bad, r0 + lane);
        epi.row(r0 + lane, present, sum);
      }
      __syncwarp();
    } else {
      // A piece [b, d) (at most 256 entries) of row a: each lane folds a
      // contiguous run of 8, then the lanes combine left to right.
      const uint32_t row = unit.a, e0 = unit.b, e1 = unit.d;
      const uint32_t slot = unit.c & 0x7fffffffu;
      const uint32_t count = e1 - e0;
      stage_products<E, S, W>(A, x, e0, count, stage, err, row);
      __syncwarp();
      Partial<E, ADD> mine{Acc<E, ADD>::of(E{}), false};
      constexpr uint32_t per = kTileEntries / 32;
      for (uint32_t k = lane * per; k < min(count, lane * per + per); k++)
        mine = join(mine, Partial<E, ADD>{Acc<E, ADD>::of(stage[k]), true});
      for (unsigned o = 1; o < 32; o <<= 1) {
        Partial<E, ADD> other = shfl_partial(mine, o);
        if ((lane & (2 * o - 1)) == 0) mine = join(mine, other);
      }
      __syncwarp();
      if (lane == 0) {
        const uint32_t row_lo = __ldg(A.off + row);
        const uint32_t deg = __ldg(A.off + row + 1) - row_lo;
        const uint32_t pieces = (deg + kPieceEntries - 1) / kPieceEntries;
        const uint32_t first = slot - (e0 - row_lo) / kPieceEntries;
        carry[slot] = mine;
        __threadfence();
        const uint32_t arrived = atomicAdd(A.counters + first, 1u);
        if (arrived == pieces - 1) {
          __threadfence();
          Partial<E, ADD> total = load_cg(carry + first);
          for (uint32_t p = 1; p < pieces; p++) total = join(total, load_cg(carry + first + p));
          A.counters[first] = 0;
          E v;
          int32_t s = total.acc.value(&v);
          if (s) raise(err, s, row);
          epi.row(row, true, v);
        }
      }
    }
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
  __device__ void row(uint32_t row, bool present, E t) {
    const E identity = Identity<E>::of(semiring_add(S));
    if (!mask_selects(w, row)) {
      if (w.replace) y[row] = identity;
      return;
    }
    if (w.accumulate < 0) {
      y[row] = present ? t : identity;
    } else if (present) {
      E out;
      int32_t s = apply_rt<E>(w.accumulate, y[row], t, &out);
      if (s) raise(err, s, row);
      else y[row] = out;
    }
  }
};

}  // namespace wc
