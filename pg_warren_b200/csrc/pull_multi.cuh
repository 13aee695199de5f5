// pull_multi.cuh — the pull kernel over P columns at once: Y = A ⊗ X for a
// row-major id_space × P operand X, walked by the same row-split schedule
// as the SpMV (pull.cuh).  It serves the batched searches (a pass of P
// sources or seed sets).
//
// The warp's lanes form 32/P groups of P; lane c of a group owns column c.
// In a tile, the groups take the tile's rows in turn and each lane folds its
// column over the row's entries in ascending order — the reference's fold
// (compute/product/kernel.rs:184-198) to the bit — with the row's targets
// loaded 32 at a time and eight rows of X gathered ahead.  A long row's
// pieces (at most 256 entries) are split between the groups as contiguous
// runs, combined left to right, and the pieces of one row combined in piece
// order by the last to finish, so only floating-point plus in rows over 256
// entries is reassociated.
#pragma once

#include "pull.cuh"

namespace wc {

// Bit i of a tombstone bitmap (NULL: no tombstones).
__device__ inline bool tomb_bit(const uint64_t* t, uint32_t i) {
  return t && ((t[i >> 6] >> (i & 63)) & 1);
}

// The schedule view of one orientation with its weights (W = void: none).
template <class W> CsrView<W> view_of(const DevCsr& csr, const void* weights) {
  return CsrView<W>{csr.offsets.as<uint32_t>(), csr.targets.as<uint32_t>(),
                    static_cast<const W*>(weights), csr.schedule.units.as<Unit>(),
                    csr.schedule.count, csr.schedule.counters.as<uint32_t>(), nullptr};
}

// Folds entries [e0, e1) of column `c` into `acc` in order (X's rows are
// `ld` elements apart; an inactive lane folds nothing).  All lanes of the
// group run the same trip count (the group shares the row).
template <class E, int S, class W, int P>
__device__ inline void fold_run(const CsrView<W>& A, const E* __restrict__ X, uint32_t e0,
                                uint32_t e1, uint32_t c, Partial<E, semiring_add(S)>& acc,
                                DeviceError* err, uint32_t row, uint32_t ld = P,
                                bool active = true) {
  constexpr int ADD = semiring_add(S);
  constexpr int U = 8;
  for (uint32_t e = e0; e < e1; e += U) {
    uint32_t j[U];
    typename EntryOf<E, S, W>::WT wv[U];
#pragma unroll
    for (int q = 0; q < U; q++) {
      if (e + q < e1) {
        j[q] = __ldg(A.tgt + e + q);
        wv[q] = EntryOf<E, S, W>::load(A, e + q);
      }
    }
    E xv[U];
#pragma unroll
    for (int q = 0; q < U; q++)
      if (active && e + q < e1) xv[q] = X[(size_t)j[q] * ld + c];
#pragma unroll
    for (int q = 0; q < U; q++) {
      if (active && e + q < e1) {
        E p;
        int32_t s = EntryOf<E, S, W>::product(wv[q], xv[q], &p);
        if (s) raise(err, s, row);
        if (acc.present) {
          E sum;
          acc.acc.value(&sum);
          s = Apply<E, ADD>::go(sum, p, &sum);
          if (s) raise(err, s, row);
          acc.acc = Acc<E, ADD>::of(sum);
        } else {
          acc.acc = Acc<E, ADD>::of(p);
          acc.present = true;
        }
      }
    }
  }
}

// Walks the schedule; `epi.cell(row, column, present, value)` is called
// once per (row, column), always by a lane whose index is column mod P, so
// an epilogue may keep per-column sums in registers.  X's rows are `ld`
// elements apart; columns >= `columns`, and columns whose bit in `mask` is
// clear, are folded by no lane (their cells still come, with unspecified
// values).  `carry` holds P partials per slot (the schedule's long-row
// pieces).
template <class E, int S, class W, int P, class Epi>
__device__ inline void pull_multi(const CsrView<W>& A, const E* __restrict__ X, Epi& epi,
                                  DeviceError* err, Partial<E, semiring_add(S)>* carry,
                                  uint32_t ld = P, uint32_t columns = P,
                                  uint32_t mask = 0xffffffffu) {
  static_assert(P >= 1 && P <= 32 && (P & (P - 1)) == 0, "P: a power of two up to 32");
  constexpr int ADD = semiring_add(S);
  constexpr uint32_t G = 32 / P;
  const unsigned lane = threadIdx.x & 31;
  const uint32_t c = lane % P, g = lane / P;
  const bool active = c < columns && ((mask >> c) & 1);
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < A.unit_count; u += warps) {
    const Unit unit = A.units[u];
    if ((unit.c >> 31) == 0) {
      for (uint32_t r = unit.a + g; r < unit.b; r += G) {
        const uint32_t lo = __ldg(A.off + r), hi = __ldg(A.off + r + 1);
        Partial<E, ADD> acc{Acc<E, ADD>::of(E{}), false};
        fold_run<E, S, W, P>(A, X, lo, hi, c, acc, err, r, ld, active);
        E v{};
        if (acc.present) acc.acc.value(&v);
        epi.cell(r, c, acc.present, v);
      }
    } else {
      const uint32_t row = unit.a, e0 = unit.b, e1 = unit.d;
      const uint32_t slot = unit.c & 0x7fffffffu;
      const uint32_t run = (kPieceEntries + G - 1) / G;
      Partial<E, ADD> mine{Acc<E, ADD>::of(E{}), false};
      const uint32_t b0 = min(e1, e0 + g * run), b1 = min(e1, e0 + (g + 1) * run);
      fold_run<E, S, W, P>(A, X, b0, b1, c, mine, err, row, ld, active);
      for (uint32_t o = P; o < 32; o <<= 1) {  // groups o/P apart: left to right
        Partial<E, ADD> other = shfl_partial(mine, o);
        if ((g & (2 * (o / P) - 1)) == 0) mine = join(mine, other);
      }
      const uint32_t row_lo = __ldg(A.off + row);
      const uint32_t deg = __ldg(A.off + row + 1) - row_lo;
      const uint32_t pieces = (deg + kPieceEntries - 1) / kPieceEntries;
      const uint32_t first = slot - (e0 - row_lo) / kPieceEntries;
      if (g == 0) carry[(size_t)slot * P + c] = mine;
      __threadfence();
      __syncwarp();
      uint32_t arrived = 0;
      if (lane == 0) arrived = atomicAdd(A.counters + first, 1u);
      arrived = __shfl_sync(0xffffffffu, arrived, 0);
      if (arrived == pieces - 1) {
        __threadfence();
        Partial<E, ADD> total = combine_pieces<E, ADD, P>(carry, first, pieces, c, g);
        if (g == 0) {
          E v;
          int32_t s = total.acc.value(&v);
          if (s) raise(err, s, row);
          epi.cell(row, c, true, v);
        }
        __syncwarp();
        if (lane == 0) A.counters[first] = 0;
      }
    }
  }
}

}  // namespace wc
