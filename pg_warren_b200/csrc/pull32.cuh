// pull32.cuh — the pull of a 32-column f64 SpMM over a CSR's row-split
// schedule, for solvers bound by the latency of their row gathers (the
// batched personalised PageRank, the PageRank adjoint).
//
// A row of the gathered operand is 256 bytes and one lane owns one column.
// A warp keeps its gathers in flight as asynchronous copies (cp.async) into
// a ring in shared memory instead of registers (16 bytes a lane, a
// half-warp an entry): a unit's entries go out 16 at a time, two groups in
// flight, while the targets, row ends and per-row
// values load into lanes.  A warp's shared memory is only its ring (8 KB),
// so as many warps fit an SM as the registers allow.  Entries are folded in
// ascending order per row, as pull_multi folds them, so each row's sum is
// the same to the bit; a long row's pieces are combined in piece order by
// the warp that brings the last of them.
//
// The solver's epilogue `Epi` provides:
//   Row                      per-row values, loaded by the tile's lane r for
//                            its row r (coalesced) and shuffled at the emit;
//   Row row(i) const         those of row i;
//   Row shfl(Row, src) const lane src's;
//   void emit(i, acc, Row)   row i's result for this lane's column;
//   bool active              whether this lane's column runs at all.
#pragma once

#include "pull.cuh"

namespace wc {

constexpr uint32_t kPull32Warps = 4;          // warps a block
constexpr uint32_t kPull32Chunk = 16;         // entries a gather group
constexpr uint32_t kPull32WarpDoubles = 1024;  // the ring: 2 groups × 16 entries × 32 columns
constexpr size_t kPull32Smem = kPull32Warps * kPull32WarpDoubles * sizeof(double);

__device__ inline void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
__device__ inline void cp_async16_ca(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ inline void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// v[i] for a register array and a run-time i (selects, no local memory).
template <class T> __device__ inline T pick8(const T (&v)[8], uint32_t i) {
  T r = v[0];
#pragma unroll
  for (uint32_t q = 1; q < 8; q++)
    if (i == q) r = v[q];
  return r;
}

// The warp's units of A's schedule (warp, warp + warps, ...): X is the
// gathered operand (n × 32), `ring` this warp's kPull32WarpDoubles.
template <class W, class Epi>
__device__ inline void pull32_units(const CsrView<W>& A, const double* __restrict__ X, Epi& epi,
                                    DeviceError* err, Partial<double, WC_OP_PLUS>* carry,
                                    double* ring) {
  constexpr int ADD = WC_OP_PLUS;
  typedef EntryOf<double, WC_PLUS_TIMES, W> Ent;
  typedef Partial<double, ADD> Part;
  typedef typename Epi::Row Row;
  const unsigned lane = threadIdx.x & 31;
  const bool active = epi.active;
  const unsigned amask = __ballot_sync(0xffffffffu, active);  // the running columns
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;

  // Folds the entry gathered into ring slot `slot` into `acc`.
  auto fold = [&](Part& acc, uint32_t slot, typename Ent::WT wv, uint32_t row) {
    if (!active) return;
    const double xv = ring[slot * 32 + lane];
    double p;
    int32_t st = Ent::product(wv, xv, &p);
    if (st) raise(err, st, row);
    if (acc.present) {
      double sum;
      acc.acc.value(&sum);
      st = Apply<double, ADD>::go(sum, p, &sum);
      if (st) raise(err, st, row);
      acc.acc = Acc<double, ADD>::of(sum);
    } else {
      acc.acc = Acc<double, ADD>::of(p);
      acc.present = true;
    }
  };

  for (uint32_t u = warp; u < A.unit_count; u += warps) {
    const Unit unit = A.units[u];
    const bool tile = (unit.c >> 31) == 0;
    const uint32_t a = unit.a;
    const uint32_t R = tile ? unit.b - unit.a : 1;
    const uint32_t base = tile ? unit.d : unit.b;
    const uint32_t count = tile ? unit.c : unit.d - unit.b;
    __syncwarp();  // every lane is done with the last unit's ring
    // Targets and weights of the unit (≤ 256 entries): entry 32·q + lane in
    // register q; per-row values of the tile: row `lane` in each lane.
    uint32_t jr[8];
    typename Ent::WT wr[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const uint32_t k = 32 * q + lane;
      jr[q] = k < count ? __ldg(A.tgt + base + k) : 0u;
      wr[q] = k < count ? Ent::load(A, base + k) : typename Ent::WT{};
    }
    uint32_t hi_l = count;
    Row row_l{};
    if (tile && lane < R) {
      hi_l = __ldg(A.off + a + lane + 1) - base;
      row_l = epi.row(a + lane);
    }
    const uint32_t chunks = (count + kPull32Chunk - 1) / kPull32Chunk;
    // Gather group q into ring half q & 1: each half-warp copies one
    // entry's row, 16 bytes (two columns) a lane, skipping column pairs
    // that do not run.
    const uint32_t half = lane >> 4, c2 = 2 * (lane & 15);
    const bool pair_runs = ((amask >> c2) & 3u) != 0;
    auto issue = [&](uint32_t q) {
      const uint32_t jw = pick8(jr, q >> 1), off = (q & 1) * kPull32Chunk;
      double* dst = ring + off * 32 + c2;
#pragma unroll
      for (uint32_t t = 0; t < kPull32Chunk; t += 2) {
        const uint32_t tt = t + half;
        const uint32_t j = __shfl_sync(0xffffffffu, jw, off + tt);
        if (pair_runs && q * kPull32Chunk + tt < count)
          cp_async16_ca(dst + tt * 32, X + (size_t)j * 32 + c2);
      }
      cp_async_commit();
    };
    if (chunks > 0) issue(0);
    Part acc{Acc<double, ADD>::of(0.0), false};
    uint32_t r = 0;
    uint32_t hi_r = __shfl_sync(0xffffffffu, hi_l, 0);
    for (uint32_t q = 0; q < chunks; q++) {
      // A lane's copies fill other lanes' columns: every lane is done with
      // the half that group q + 1 refills (group q - 1's) before it is.
      __syncwarp();
      if (q + 1 < chunks) {
        issue(q + 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncwarp();
      const uint32_t n_q = min(kPull32Chunk, count - q * kPull32Chunk);
      const typename Ent::WT ww = pick8(wr, q >> 1);
      const uint32_t k0 = q * kPull32Chunk;
      if (n_q == kPull32Chunk && k0 + kPull32Chunk <= hi_r) {
        // No row ends inside this chunk: its entries all fold into the
        // current row, in order, with no boundary test between them.
        const uint32_t row = tile ? a + r : a;
#pragma unroll
        for (uint32_t t = 0; t < kPull32Chunk; t++) {
          const typename Ent::WT wv = (typename Ent::WT)__shfl_sync(0xffffffffu, ww, (k0 + t) & 31);
          fold(acc, (q & 1) * kPull32Chunk + t, wv, row);
        }
        continue;
      }
      // Otherwise row by row: emit the rows that end before entry t, then
      // fold the chunk's entries of the current row with no test between.
      for (uint32_t t = 0; t < n_q;) {
        while (k0 + t >= hi_r) {  // rows ending before entry k0 + t (tiles only)
          epi.emit(a + r, acc, epi.shfl(row_l, r));
          acc = Part{Acc<double, ADD>::of(0.0), false};
          r++;
          hi_r = __shfl_sync(0xffffffffu, hi_l, r);
        }
        const uint32_t end = min(n_q, hi_r - k0);
        const uint32_t row = tile ? a + r : a;
        for (; t < end; t++) {
          const typename Ent::WT wv = (typename Ent::WT)__shfl_sync(0xffffffffu, ww, (k0 + t) & 31);
          fold(acc, (q & 1) * kPull32Chunk + t, wv, row);
        }
      }
    }
    if (chunks == 0) {
      cp_async_wait<0>();
      __syncwarp();
    }
    if (tile) {
      for (; r < R; r++) {
        epi.emit(a + r, acc, epi.shfl(row_l, r));
        acc = Part{Acc<double, ADD>::of(0.0), false};
      }
      continue;
    }
    // A piece of a long row: its partial in the carry slot; the warp that
    // brings the row's last piece combines the pieces in order and emits.
    const uint32_t row = a, slot = unit.c & 0x7fffffffu;
    const uint32_t row_lo = __ldg(A.off + row);
    const uint32_t deg = __ldg(A.off + row + 1) - row_lo;
    const uint32_t pieces = (deg + kPieceEntries - 1) / kPieceEntries;
    const uint32_t first = slot - (base - row_lo) / kPieceEntries;
    carry[(size_t)slot * 32 + lane] = acc;
    __threadfence();
    __syncwarp();
    uint32_t arrived = 0;
    if (lane == 0) arrived = atomicAdd(A.counters + first, 1u);
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived == pieces - 1) {
      __threadfence();
      const Part total = combine_pieces<double, ADD, 32>(carry, first, pieces, lane, 0);
      epi.emit(row, total, epi.row(row));
      __syncwarp();
      if (lane == 0) A.counters[first] = 0;
    }
  }
}

}  // namespace wc
