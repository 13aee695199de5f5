// batched_minplus32.cu — the batched min-plus searches (wc_minplus_batched)
// on 32-bit distances, for the versions where no distance can leave the
// 32-bit range: every weight is an i32 (or the version is unweighted) and
// max|w| × the largest cap < 2^30.  Every value the i64 loop
// (compute_sql/library/sssp_vector.sql:14-66 over i64) computes then fits,
// no i64 overflow can occur, and the i64 identity (i64::MAX, which absorbs
// plus) maps to i32::MAX: the distances and the per-column iteration counts
// are the i64 loop's.
//
// A pass runs P = 32 or 64 columns; a row's P distances are spread over
// LPR = P/4 lanes holding four each (16-byte accesses).  An iteration reads
// the previous iterate only (next = min(x, Aᵀ ⊗ x)); after iteration t every
// row holds x_i ≤ x_j + w for the values of iteration t-1, so iteration t+1
// folds only the entries whose source row fell at t (a bitmap).  Rows that
// fall are written to a second buffer and copied in by a short kernel after
// the iteration.  Long rows' pieces take the minimum into per-row global
// accumulators; the last piece to arrive settles the row.
#include <algorithm>
#include <string>

#include "batched.h"
#include "operand.h"
#include "semiring.cuh"

namespace wc {

constexpr int32_t kInf32 = INT32_MAX;

struct Mp32 {
  uint32_t n;
  const uint32_t* off;
  const uint32_t* tgt;
  const int32_t* w;    // NULL: unweighted (every weight 1)
  const Unit* units;
  uint32_t unit_count;
  uint32_t* counters;  // per long row (first slot), left zero
  int32_t* nacc;       // P per long row (first slot), left at kInf32
  int32_t* x;          // n × P: the current iterate
  int32_t* next;       // n × P: the rows that fell this iteration
  uint32_t* fell_rows[2];
  const uint32_t* caps;  // P (this pass)
  const uint32_t* cols;  // P: the call's column of each pass column
  uint32_t k;
  uint32_t* running;   // P/32 words: columns still iterating
  uint32_t* fell;      // P/32 words: columns whose distances fell this iteration
  uint32_t* iterations;  // the call's, indexed by cols
};

__device__ inline int32_t add_absorbing(int32_t x, int32_t w) { return x == kInf32 ? kInf32 : x + w; }

template <int P> struct Mp32Smem {
  int32_t acc[32 * P];
  uint32_t hitj[kTileEntries];
  int32_t hitw[kTileEntries];
  uint8_t hitr[kTileEntries];
  uint8_t rowof[kTileEntries];
};

__global__ void mp32_fill_kernel(int32_t* p, uint64_t count, int32_t v) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < count;
       q += (uint64_t)gridDim.x * blockDim.x)
    p[q] = v;
}

template <int P>
__global__ void mp32_seed_kernel(Mp32 s, const uint64_t* sources) {
  const size_t total = (size_t)s.n * P;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x)
    s.x[q] = kInf32;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < (s.n + 31) / 32;
       q += (size_t)gridDim.x * blockDim.x) {
    s.fell_rows[0][q] = 0;
    s.fell_rows[1][q] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x < P / 32) {
    uint32_t run = 0;
    for (uint32_t b = 0; b < 32; b++) {
      const uint32_t c = 32 * threadIdx.x + b;
      if (c < s.k && s.caps[c] > 0) run |= 1u << b;
    }
    s.running[threadIdx.x] = run;
    s.fell[threadIdx.x] = 0;
  }
  if (blockIdx.x == 0)
    for (uint32_t c = threadIdx.x; c < s.k; c += blockDim.x) s.iterations[s.cols[c]] = 0;
}

template <int P>
__global__ void mp32_sources_kernel(Mp32 s, const uint64_t* sources) {
  for (uint32_t c = threadIdx.x; c < s.k; c += blockDim.x) {
    const uint32_t node = (uint32_t)sources[c];
    s.x[(size_t)node * P + c] = 0;
    atomicOr(s.fell_rows[0] + (node >> 5), 1u << (node & 31));
  }
}

// One iteration over the reverse CSR's schedule.
template <int P>
__global__ void __launch_bounds__(256, 3) mp32_iter_kernel(Mp32 s, uint32_t it) {
  constexpr uint32_t LPR = P / 4;       // lanes a row
  constexpr uint32_t G = 32 / LPR;      // rows (or gathered rows) a warp instruction covers
  constexpr uint32_t GM = LPR == 32 ? 0xffffffffu : (1u << LPR) - 1;
  constexpr int Q = kTileEntries / 32;
  constexpr int U = 8;
  constexpr uint32_t VR = kTileRows / G;
  bool any_running = false;
  for (uint32_t q = 0; q < P / 32; q++) any_running |= s.running[q] != 0;
  if (!any_running) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Mp32Smem<P>& sm = reinterpret_cast<Mp32Smem<P>*>(smem_raw)[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31;
  const unsigned sub = lane / LPR, q = lane % LPR;
  const uint32_t c0 = q * 4;  // this lane's four columns
  const unsigned gmask = GM << (sub * LPR);
  const uint32_t run4 = (s.running[c0 >> 5] >> (c0 & 31)) & 0xFu;  // running bits of c0..c0+3
  const uint32_t* fell_cur = s.fell_rows[it & 1];
  uint32_t* fell_next = s.fell_rows[(it + 1) & 1];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  uint32_t fell_cols = 0;  // bits of this lane's four columns that fell

  // new = min(old, got) for running columns; f: the columns that fell.
  auto settle = [&](uint32_t i, const int4& got, int4& nv) -> uint32_t {
    const int4 old = *reinterpret_cast<const int4*>(s.x + (size_t)i * P + c0);
    nv = old;
    if ((run4 & 1) && got.x < old.x) nv.x = got.x;
    if ((run4 & 2) && got.y < old.y) nv.y = got.y;
    if ((run4 & 4) && got.z < old.z) nv.z = got.z;
    if ((run4 & 8) && got.w < old.w) nv.w = got.w;
    return (nv.x < old.x ? 1u : 0u) | (nv.y < old.y ? 2u : 0u) | (nv.z < old.z ? 4u : 0u) |
           (nv.w < old.w ? 8u : 0u);
  };

  for (uint32_t u = warp; u < s.unit_count; u += warps) {
    const Unit unit = s.units[u];
    const bool tile = (unit.c >> 31) == 0;
    const uint32_t r0 = unit.a;
    const uint32_t R = tile ? unit.b - unit.a : 1;
    uint32_t base, count;
    if (tile) {
      uint32_t lo = 0, hi = 0;
      if (lane < R) {
        lo = __ldg(s.off + r0 + lane);
        hi = __ldg(s.off + r0 + lane + 1);
      }
      base = unit.d;
      count = unit.c;
      for (uint32_t k = lo - base; k < hi - base; k++) sm.rowof[k] = (uint8_t)lane;
      for (uint32_t x = lane * 4; x < R * P; x += 128)
        *reinterpret_cast<int4*>(&sm.acc[x]) = make_int4(kInf32, kInf32, kInf32, kInf32);
    } else {
      base = unit.b;
      count = unit.d - unit.b;
    }
    __syncwarp();
    // The hits: entries whose source row fell in the previous iteration.
    uint32_t H = 0;
    {
      uint32_t jv[Q];
#pragma unroll
      for (int qq = 0; qq < Q; qq++) {
        const uint32_t k = lane + 32 * qq;
        jv[qq] = k < count ? __ldcs(s.tgt + base + k) : 0u;
      }
#pragma unroll
      for (int qq = 0; qq < Q; qq++) {
        const uint32_t k = lane + 32 * qq;
        const bool hit = k < count && ((fell_cur[jv[qq] >> 5] >> (jv[qq] & 31)) & 1);
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
          const uint32_t pos = H + __popc(m & ((1u << lane) - 1));
          sm.hitj[pos] = jv[qq];
          sm.hitw[pos] = s.w ? __ldg(s.w + base + k) : 1;
          sm.hitr[pos] = tile ? sm.rowof[k] : (uint8_t)0;
        }
        H += __popc(m);
      }
    }
    __syncwarp();
    // Gather: group g takes hits [g·H/G, (g+1)·H/G) in order; a row's hits
    // are consecutive, so their minima stay in registers until the row
    // changes.
    int4 run = make_int4(kInf32, kInf32, kInf32, kInf32);
    if (H) {
      const uint32_t per = (H + G - 1) / G;
      const uint32_t h_lo = min(H, sub * per), h_hi = min(H, sub * per + per);
      uint32_t cur = h_lo < h_hi ? sm.hitr[h_lo] : 0u;
      for (uint32_t h0 = h_lo; h0 < h_hi; h0 += U) {
        int4 val[U];
        int32_t wv[U];
        uint32_t rr[U];
#pragma unroll
        for (int x = 0; x < U; x++) {
          const uint32_t h = h0 + x;
          rr[x] = cur;
          wv[x] = 0;
          val[x] = make_int4(kInf32, kInf32, kInf32, kInf32);
          if (h < h_hi) {
            val[x] = __ldg(reinterpret_cast<const int4*>(s.x + (size_t)sm.hitj[h] * P + c0));
            wv[x] = sm.hitw[h];
            rr[x] = sm.hitr[h];
          }
        }
#pragma unroll
        for (int x = 0; x < U; x++) {
          if (rr[x] != cur) {
            if (tile) {
              int32_t* a = &sm.acc[cur * P + c0];
              if (run.x != kInf32) atomicMin(a, run.x);
              if (run.y != kInf32) atomicMin(a + 1, run.y);
              if (run.z != kInf32) atomicMin(a + 2, run.z);
              if (run.w != kInf32) atomicMin(a + 3, run.w);
            }
            run = make_int4(kInf32, kInf32, kInf32, kInf32);
            cur = rr[x];
          }
          run.x = min(run.x, add_absorbing(val[x].x, wv[x]));
          run.y = min(run.y, add_absorbing(val[x].y, wv[x]));
          run.z = min(run.z, add_absorbing(val[x].z, wv[x]));
          run.w = min(run.w, add_absorbing(val[x].w, wv[x]));
        }
      }
      if (tile) {
        int32_t* a = &sm.acc[cur * P + c0];
        if (run.x != kInf32) atomicMin(a, run.x);
        if (run.y != kInf32) atomicMin(a + 1, run.y);
        if (run.z != kInf32) atomicMin(a + 2, run.z);
        if (run.w != kInf32) atomicMin(a + 3, run.w);
      }
    }
    __syncwarp();
    if (tile) {
#pragma unroll
      for (uint32_t x = 0; x < VR; x++) {
        if (x * G >= R) break;
        const uint32_t r = x * G + sub;
        uint32_t f = 0;
        int4 nv = make_int4(0, 0, 0, 0);
        if (r < R) {
          const int4 got = *reinterpret_cast<const int4*>(&sm.acc[r * P + c0]);
          f = settle(r0 + r, got, nv);
        }
        if (__ballot_sync(0xffffffffu, f != 0) & gmask) {
          *reinterpret_cast<int4*>(s.next + (size_t)(r0 + r) * P + c0) = nv;
          if (q == 0) atomicOr(fell_next + ((r0 + r) >> 5), 1u << ((r0 + r) & 31));
        }
        fell_cols |= f;
      }
      __syncwarp();
    } else {
      // The groups' minima, then into the row's global accumulator.
#pragma unroll
      for (uint32_t o = LPR; o < 32; o <<= 1) {
        run.x = min(run.x, __shfl_xor_sync(0xffffffffu, run.x, o));
        run.y = min(run.y, __shfl_xor_sync(0xffffffffu, run.y, o));
        run.z = min(run.z, __shfl_xor_sync(0xffffffffu, run.z, o));
        run.w = min(run.w, __shfl_xor_sync(0xffffffffu, run.w, o));
      }
      const uint32_t row = unit.a, slot = unit.c & 0x7fffffffu;
      const uint32_t row_lo = __ldg(s.off + row);
      const uint32_t deg = __ldg(s.off + row + 1) - row_lo;
      const uint32_t pieces = (deg + kPieceEntries - 1) / kPieceEntries;
      const uint32_t first = slot - (unit.b - row_lo) / kPieceEntries;
      int32_t* na = s.nacc + (size_t)first * P + c0;
      if (sub == 0) {
        if (run.x != kInf32) atomicMin(na, run.x);
        if (run.y != kInf32) atomicMin(na + 1, run.y);
        if (run.z != kInf32) atomicMin(na + 2, run.z);
        if (run.w != kInf32) atomicMin(na + 3, run.w);
      }
      __threadfence();
      __syncwarp();
      uint32_t arrived = 0;
      if (lane == 0) arrived = atomicAdd(s.counters + first, 1u);
      arrived = __shfl_sync(0xffffffffu, arrived, 0);
      if (arrived == pieces - 1) {
        __threadfence();
        uint32_t f = 0;
        int4 nv = make_int4(0, 0, 0, 0);
        if (sub == 0) {
          const int4 got = make_int4(__ldcg(na), __ldcg(na + 1), __ldcg(na + 2), __ldcg(na + 3));
          *reinterpret_cast<int4*>(na) = make_int4(kInf32, kInf32, kInf32, kInf32);
          f = settle(row, got, nv);
        }
        if (__ballot_sync(0xffffffffu, f != 0)) {
          if (sub == 0) *reinterpret_cast<int4*>(s.next + (size_t)row * P + c0) = nv;
          if (lane == 0) atomicOr(fell_next + (row >> 5), 1u << (row & 31));
        }
        fell_cols |= f;
        if (lane == 0) s.counters[first] = 0;
      }
    }
  }
  // The columns that fell: lanes q of every group hold columns 4q..4q+3.
#pragma unroll
  for (uint32_t o = LPR; o < 32; o <<= 1) fell_cols |= __shfl_xor_sync(0xffffffffu, fell_cols, o);
  if (sub == 0 && fell_cols) atomicOr(s.fell + (c0 >> 5), fell_cols << (c0 & 31));
}

// Copies the rows that fell into the iterate; clears the bitmap the
// iteration read (the next iteration writes it).
template <int P>
__global__ void mp32_apply_kernel(Mp32 s, uint32_t it) {
  const uint32_t* fell_next = s.fell_rows[(it + 1) & 1];
  uint32_t* fell_cur = s.fell_rows[it & 1];
  const uint32_t words = (s.n + 31) / 32;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = warp; t < words; t += warps) {
    uint32_t bits = fell_next[t];
    if (lane == 0) fell_cur[t] = 0;
    while (bits) {
      const uint32_t i = 32 * t + __ffs(bits) - 1;
      bits &= bits - 1;
      for (uint32_t c = 4 * lane; c < P; c += 128)
        *reinterpret_cast<int4*>(s.x + (size_t)i * P + c) =
            *reinterpret_cast<const int4*>(s.next + (size_t)i * P + c);
    }
  }
}

// After iteration `it`: a running column whose distances did not fall
// stops with it + 1 iterations; one at its cap stops too.
template <int P>
__global__ void mp32_control_kernel(Mp32 s, uint32_t it) {
  const uint32_t wq = threadIdx.x;
  if (wq >= P / 32) return;
  uint32_t run = s.running[wq], fell = s.fell[wq];
  for (uint32_t b = 0; b < 32; b++) {
    const uint32_t c = 32 * wq + b;
    if (!((run >> b) & 1)) continue;
    s.iterations[s.cols[c]] = it + 1;
    if (!((fell >> b) & 1) || it + 1 >= s.caps[c]) run &= ~(1u << b);
  }
  s.running[wq] = run;
  s.fell[wq] = 0;
}

// out[cols[c] * n + i] = x[i * P + c] widened to i64 (i32::MAX → i64::MAX).
template <int P>
__global__ void mp32_out_kernel(const int32_t* x, uint32_t n, uint32_t k, const uint32_t* cols,
                                int64_t* out) {
  __shared__ int32_t tile[32][P + 1];
  const uint32_t tiles = (n + 31) / 32;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint32_t i0 = t * 32;
    for (uint32_t q = threadIdx.x; q < 32 * P; q += blockDim.x) {
      const uint32_t r = q / P, c = q % P;
      if (i0 + r < n) tile[r][c] = x[(size_t)(i0 + r) * P + c];
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < 32 * k; q += blockDim.x) {
      const uint32_t c = q / 32, r = q % 32;
      if (i0 + r < n) {
        const int32_t v = tile[r][c];
        out[(size_t)cols[c] * n + i0 + r] = v == kInf32 ? INT64_MAX : (int64_t)v;
      }
    }
    __syncthreads();
  }
}

template <int P>
wc_status mp32_pass(Ctx& ctx, const uint64_t* sources, const uint32_t* caps, const uint32_t* cols,
                    uint32_t k, uint32_t max_cap, int64_t* out, uint32_t* iterations,
                    uint32_t blocks_per_sm) {
  wc_version* v = ctx.v;
  const uint32_t n = (uint32_t)v->n;
  const uint64_t words = (n + 31) / 32;
  DevBuf *xb, *stb, *nb;
  WC_TRY(ctx.scratch(POOL_BATCH_0, (uint64_t)n * P * 4 * 2, &xb));
  WC_TRY(ctx.scratch(POOL_BATCH_1, 256 + 2 * words * 4, &stb));
  // Long-row accumulators, kept at kInf32 between iterations (and calls).
  const uint64_t nacc_bytes = (uint64_t)std::max<uint32_t>(v->rev.schedule.slots, 1) * 64 * 4;
  WC_TRY(ctx.scratch(POOL_MINPLUS32_NACC, nacc_bytes, &nb));
  Mp32 s{};
  const DevCsr& csc = v->rev;
  s.n = n;
  s.off = csc.offsets.as<uint32_t>();
  s.tgt = csc.targets.as<uint32_t>();
  s.w = v->weighted ? csc.iweights.as<int32_t>() : nullptr;
  s.units = csc.schedule.units.as<Unit>();
  s.unit_count = csc.schedule.count;
  s.counters = csc.schedule.counters.as<uint32_t>();
  s.nacc = nb->as<int32_t>();
  s.x = xb->as<int32_t>();
  s.next = s.x + (size_t)n * P;
  s.running = stb->as<uint32_t>();
  s.fell = s.running + 8;
  s.fell_rows[0] = s.running + 64;
  s.fell_rows[1] = s.fell_rows[0] + words;
  s.caps = caps;
  s.cols = cols;
  s.k = k;
  s.iterations = iterations;
  cudaStream_t st = ctx.stream;
  note_launch(), mp32_seed_kernel<P><<<max_blocks(4), 256, 0, st>>>(s, sources);
  note_launch(), mp32_sources_kernel<P><<<1, 128, 0, st>>>(s, sources);
  const size_t smem = 8 * sizeof(Mp32Smem<P>);
  static const cudaError_t attr = cudaFuncSetAttribute(
      mp32_iter_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (attr != cudaSuccess) return cuda_status(attr, ctx.detail, "min-plus kernel attributes");
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(
      max_blocks((int)blocks_per_sm), (csc.schedule.count + 7) / 8));
  const uint32_t apply_grid = std::max<uint32_t>(1, std::min<uint32_t>(
      max_blocks(8), (uint32_t)((words + 7) / 8)));
  for (uint32_t it = 0; it < max_cap; it++) {
    note_launch(), mp32_iter_kernel<P><<<grid, 256, smem, st>>>(s, it);
    note_launch(), mp32_apply_kernel<P><<<apply_grid, 256, 0, st>>>(s, it);
    note_launch(), mp32_control_kernel<P><<<1, 32, 0, st>>>(s, it);
  }
  note_launch(), mp32_out_kernel<P><<<max_blocks(2), 256, 0, st>>>(s.x, n, k, cols, out);
  return cuda_status(cudaGetLastError(), ctx.detail, "batched min-plus pass");
}

// The pass's scratch, acquired before a pass is captured; a fresh long-row
// accumulator buffer is set to kInf32 once.
wc_status mp32_reserve(Ctx& ctx, uint32_t P) {
  wc_version* v = ctx.v;
  DevBuf* b;
  WC_TRY(ctx.scratch(POOL_BATCH_0, (uint64_t)v->n * P * 4 * 2, &b));
  WC_TRY(ctx.scratch(POOL_BATCH_1, 256 + 2 * ((v->n + 31) / 32) * 4, &b));
  const uint64_t nacc_bytes = (uint64_t)std::max<uint32_t>(v->rev.schedule.slots, 1) * 64 * 4;
  const bool fresh = v->pool[POOL_MINPLUS32_NACC].bytes < nacc_bytes;
  WC_TRY(ctx.scratch(POOL_MINPLUS32_NACC, nacc_bytes, &b));
  if (fresh) {
    note_launch(), mp32_fill_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(
        b->as<int32_t>(), b->bytes / 4, kInf32);
    WC_CUDA(cudaGetLastError(), ctx.detail);
  }
  return WC_OK;
}

Mp32Fn mp32_for(uint32_t p) { return p <= 32 ? mp32_pass<32> : mp32_pass<64>; }

}  // namespace wc
