// batched_ppr.cu — wc_ppr_batched: many personalised PageRanks (one per
// seed set) run as one SpMM over P columns (pull_multi.cuh).  No reference
// counterpart; each set computes what compute/pagerank/mod.rs:96-287
// computes for a seed vector of 1 on the set (personalisation 1/|set|).
//
// The P columns are slots, not a fixed pass: a slot whose set stops (its
// delta under live × tol, pagerank/mod.rs:144-148, or max_iter) has its
// ranks copied out after that iteration and takes the next set at once,
// starting from the uniform start vector.  Sets stop after very different
// iteration counts (on R-MAT 22 from a few to about three times the mean),
// so a fixed pass would run most of its columns idle; the slots keep them
// all working until the sets run out.  A set's arithmetic does not depend
// on its slot or on what the other slots run: its result is the one it
// would get alone in a pass.
//
// One global iteration is three launches: the iteration (the pull over the
// reverse CSR's schedule, the rank update of the running columns and, in
// the last block, the stop test and the hand-out of new sets), the row
// pass for the slots that stopped (ranks out, start vector in, membership
// bits cleared) and the membership bits of the new sets.  A chunk of
// iterations is captured once as a CUDA graph and replayed; the device
// reports its progress in host-mapped words and the host keeps at most two
// chunks queued beyond it, stopping once every set has finished.
#include <algorithm>
#include <chrono>
#include <string>
#include <thread>

#include "batched.h"
#include "columns.cuh"
#include "operand.h"
#include "pagerank.h"
#include "pull32.cuh"
#include "pull_multi.cuh"
#include "sqlfloat.cuh"
#include "upload.h"

namespace wc {

constexpr uint32_t kNoSet = 0xffffffffu;
constexpr uint32_t kChunkIterations = 4;

// The device control block of a streaming run (one per call).
struct PprCtl {
  uint32_t running;   // slots whose set runs
  uint32_t finished;  // slots whose set stopped in the last iteration
  uint32_t refilled;  // slots that took a new set in the last iteration
  uint32_t g;         // global iterations run
  uint32_t next;      // the next set to hand out
  unsigned counter;   // reduce_columns' arrival counter
  uint32_t pad[2];
  uint32_t slot_set[32], fin_set[32], slot_it[32];
  double dangling[32], share[32];
  double d0;  // the start vector's dangling mass (the same for every set)
};

// The per-node state (x, msg, out, member, tomb) is kept in the version's
// locality order (locality.cu), the order of the CSC the iterations pull
// over; the sets come in and the ranks go out in dense ids.
struct PprStream {
  uint32_t n, width, max_iter;
  double* x[2];    // n × P
  double* msg[2];  // n × P
  const double* out;       // out-weights
  uint32_t* member;        // n: bit c set if row k's node is in slot c's set
  const double* shares;    // per set: 1 / |set|
  const uint64_t* nodes;   // the sets, CSR
  const uint64_t* offsets;
  const uint64_t* tomb;
  const uint32_t* perm;    // dense id -> row of the locality order
  double start, damping, teleport, threshold;
  bool has_tol;
  PprCtl* ctl;
  double* partials;     // blocks × P × 2
  double* ranks;        // width × n
  uint32_t* iterations;  // per set
  uint32_t* pace;        // host-mapped: [0] global iterations done, [1] every set finished
  DeviceError* err;
};

__device__ inline double ppr_spread(double x, double out, double* msg, DeviceError* err, uint32_t i) {
  if (sql_cmp_f(out, 0.0) > 0) {
    double m;
    int32_t s = sql_float<F_DIV>(x, out, &m);
    if (s) raise(err, s, i);
    *msg = m;
    return 0.0;
  }
  *msg = 0.0;
  return x;
}

// The rank update of one (row, running column): pagerank/mod.rs:201-282
// with the personalisation p = share on the set's nodes, 0 elsewhere.
template <int P> struct PprEpi {
  const PprStream* s;
  int cur;
  uint32_t run;
  double dangling_in, share;  // this lane's column
  double delta, dangling_out;
  __device__ void cell(uint32_t i, uint32_t c, bool present, double y) {
    if (!((run >> c) & 1)) return;
    const PprStream& st = *s;
    const size_t at = (size_t)i * P + c;
    const double old = st.x[cur][at];
    if (!present) y = 0.0;
    double next = 0.0;
    if (!tomb_bit(st.tomb, i)) {
      const double p = ((st.member[i] >> c) & 1) ? share : 0.0;
      double dp, flowed, a, b;
      int32_t e = sql_float<F_MUL>(dangling_in, p, &dp);
      if (!e) e = sql_float<F_ADD>(y, dp, &flowed);
      if (!e) e = sql_float<F_MUL>(st.damping, flowed, &a);
      if (!e) e = sql_float<F_MUL>(st.teleport, p, &b);
      if (!e) e = sql_float<F_ADD>(a, b, &next);
      if (e) raise(st.err, e, i);
    }
    delta += fabs(next - old);
    st.x[cur ^ 1][at] = next;
    dangling_out += ppr_spread(next, st.out[i], &st.msg[cur ^ 1][at], st.err, i);
  }
};

// The start vector in every column of buffer 0, its dangling mass, and the
// first min(width, P) sets in slots 0.. (their membership bits follow in
// ppr_members_kernel).
template <int P>
__global__ void ppr_init_kernel(PprStream s) {
  double none = 0.0, dangling = 0.0;
  const unsigned c = threadIdx.x % P;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / P; i < s.n;
       i += gridDim.x * blockDim.x / P) {
    const size_t at = (size_t)i * P + c;
    const double x = tomb_bit(s.tomb, i) ? 0.0 : s.start;
    s.x[0][at] = x;
    dangling += ppr_spread(x, s.out[i], &s.msg[0][at], s.err, i);
  }
  PprCtl* ctl = s.ctl;
  if (reduce_columns<P>(none, dangling, s.partials, &ctl->counter)) {
    // Threads q < P hold column q's total; every column's is the same.
    const uint32_t q = threadIdx.x;
    const uint32_t k = min(s.width, (uint32_t)P);
    if (q < 32) {
      ctl->slot_it[q] = 0;
      ctl->slot_set[q] = q < k ? q : kNoSet;
      ctl->share[q] = q < k ? s.shares[q] : 0.0;
    }
    if (q < P) ctl->dangling[q] = dangling;
    if (q == 0) {
      ctl->d0 = dangling;
      const uint32_t mask = k == 32 ? 0xffffffffu : (1u << k) - 1;
      ctl->running = mask;
      ctl->refilled = mask;
      ctl->finished = 0;
      ctl->g = 0;
      ctl->next = k;
    }
  }
}

// The last block's step after an iteration (threads q < P hold slot q's
// delta and dangling mass): each running slot's stop test
// (pagerank/mod.rs:144-148), then the next sets to the stopped slots in slot
// order, and the progress report.
template <int P>
__device__ inline void ppr_control(const PprStream& s, uint32_t run, uint32_t g, double delta,
                                   double dangling) {
  PprCtl* ctl = s.ctl;
  __shared__ uint32_t stopped;
  if (threadIdx.x == 0) stopped = 0;
  __syncthreads();
  const uint32_t q = threadIdx.x;
  if (q < P && ((run >> q) & 1)) {
    const uint32_t its = ctl->slot_it[q] + 1;
    ctl->slot_it[q] = its;
    ctl->dangling[q] = dangling;
    if (its >= s.max_iter || (s.has_tol && sql_cmp_f(delta, s.threshold) < 0)) {
      s.iterations[ctl->slot_set[q]] = its;
      atomicOr(&stopped, 1u << q);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t refilled = 0;
    for (uint32_t b = stopped; b; b &= b - 1) {
      const uint32_t slot = __ffs(b) - 1;
      ctl->fin_set[slot] = ctl->slot_set[slot];
      const uint32_t nx = ctl->next;
      if (nx < s.width) {
        ctl->next = nx + 1;
        ctl->slot_set[slot] = nx;
        ctl->share[slot] = s.shares[nx];
        ctl->dangling[slot] = ctl->d0;
        ctl->slot_it[slot] = 0;
        refilled |= 1u << slot;
      } else {
        ctl->slot_set[slot] = kNoSet;
      }
    }
    const uint32_t now = (run & ~stopped) | refilled;
    ctl->running = now;
    ctl->finished = stopped;
    ctl->refilled = refilled;
    ctl->g = g + 1;
    if (s.pace) {
      volatile uint32_t* pace = s.pace;
      pace[1] = now == 0;
      pace[0] = g + 1;
    }
  }
}

// One global iteration over the running slots (P = 8 or 16: pull_multi).
template <int P, class W>
__global__ void __launch_bounds__(256) ppr_iter_kernel(CsrView<W> A, PprStream s,
                                                       Partial<double, WC_OP_PLUS>* carry) {
  PprCtl* ctl = s.ctl;
  const uint32_t run = *(volatile uint32_t*)&ctl->running;
  if (!run) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl->finished = 0;
      ctl->refilled = 0;
    }
    return;
  }
  const uint32_t g = *(volatile uint32_t*)&ctl->g;
  const int cur = g & 1;
  const unsigned c = threadIdx.x % P;
  PprEpi<P> epi{&s, cur, run, ctl->dangling[c], ctl->share[c], 0.0, 0.0};
  pull_multi<double, WC_PLUS_TIMES, W, P>(A, s.msg[cur], epi, s.err, carry, P, P, run);
  double delta = epi.delta, dangling = epi.dangling_out;
  if (reduce_columns<P>(delta, dangling, s.partials, &ctl->counter))
    ppr_control<P>(s, run, g, delta, dangling);
}

// ------------------------------------------------------ the 32-slot pull
// With 32 slots the iteration is pull32_units (pull32.cuh) with the rank
// update as its epilogue; it is bound by instruction issue, not bandwidth.

// The rank update of row i for this lane's slot (pagerank/mod.rs:201-282).
struct PprEpi32 {
  struct Row {
    uint32_t mem;
    double out;
    bool dead;
  };
  const PprStream* s;
  const double* XO;
  double* XN;
  double* MN;
  double dangling_in, share;
  double delta = 0.0, dangling_out = 0.0;
  bool active;
  __device__ Row row(uint32_t i) const {
    return Row{s->member[i], s->out[i], tomb_bit(s->tomb, i)};
  }
  __device__ Row shfl(const Row& r, uint32_t src) const {
    return Row{__shfl_sync(0xffffffffu, r.mem, src), __shfl_sync(0xffffffffu, r.out, src),
               __shfl_sync(0xffffffffu, r.dead, src) != 0};
  }
  __device__ void emit(uint32_t i, const Partial<double, WC_OP_PLUS>& acc, const Row& r) {
    if (!active) return;
    const unsigned lane = threadIdx.x & 31;
    const PprStream& st = *s;
    const double old = XO[(size_t)i * 32 + lane];
    double y = 0.0;
    if (acc.present) acc.acc.value(&y);
    double next = 0.0;
    if (!r.dead) {
      const double p = ((r.mem >> lane) & 1) ? share : 0.0;
      double dp, flowed, a, b;
      int32_t e = sql_float<F_MUL>(dangling_in, p, &dp);
      if (!e) e = sql_float<F_ADD>(y, dp, &flowed);
      if (!e) e = sql_float<F_MUL>(st.damping, flowed, &a);
      if (!e) e = sql_float<F_MUL>(st.teleport, p, &b);
      if (!e) e = sql_float<F_ADD>(a, b, &next);
      if (e) raise(st.err, e, i);
    }
    delta += fabs(next - old);
    XN[(size_t)i * 32 + lane] = next;
    dangling_out += ppr_spread(next, r.out, &MN[(size_t)i * 32 + lane], st.err, i);
  }
};

template <class W>
__global__ void __launch_bounds__(kPull32Warps * 32, 5)
    ppr_iter32_kernel(CsrView<W> A, PprStream s, Partial<double, WC_OP_PLUS>* carry) {
  PprCtl* ctl = s.ctl;
  const uint32_t run = *(volatile uint32_t*)&ctl->running;
  if (!run) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl->finished = 0;
      ctl->refilled = 0;
    }
    return;
  }
  extern __shared__ __align__(16) double ppr_smem[];
  const uint32_t g = *(volatile uint32_t*)&ctl->g;
  const int cur = g & 1;
  const unsigned lane = threadIdx.x & 31;
  PprEpi32 epi{&s, s.x[cur], s.x[cur ^ 1], s.msg[cur ^ 1], ctl->dangling[lane], ctl->share[lane]};
  epi.active = (run >> lane) & 1;
  pull32_units<W>(A, s.msg[cur], epi, s.err, carry,
                  ppr_smem + (threadIdx.x >> 5) * kPull32WarpDoubles);
  double delta = epi.delta, dangling_out = epi.dangling_out;
  if (reduce_columns<32>(delta, dangling_out, s.partials, &ctl->counter))
    ppr_control<32>(s, run, g, delta, dangling_out);
}

// After an iteration: the stopped slots' ranks go out to their sets' rows,
// the refilled slots get the start vector, and the stopped slots'
// membership bits are cleared.
template <int P>
__global__ void ppr_rows_kernel(PprStream s) {
  const PprCtl* ctl = s.ctl;
  const uint32_t F = *(volatile const uint32_t*)&ctl->finished;
  if (!F) return;
  const uint32_t R = *(volatile const uint32_t*)&ctl->refilled;
  const int nb = ctl->g & 1;  // the buffer the last iteration wrote
  // A thread per dense id i (the ranks leave in dense-id order), its state
  // at row k of the locality order.
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
    const uint32_t k = s.perm[i];
    const uint32_t m = s.member[k];
    if (m & F) s.member[k] = m & ~F;
    for (uint32_t b = F; b; b &= b - 1) {
      const uint32_t c = __ffs(b) - 1;
      s.ranks[(size_t)ctl->fin_set[c] * s.n + i] = s.x[nb][(size_t)k * P + c];
    }
    if (R) {
      const double x0 = tomb_bit(s.tomb, k) ? 0.0 : s.start;
      double m0;
      ppr_spread(x0, s.out[k], &m0, s.err, i);
      for (uint32_t b = R; b; b &= b - 1) {
        const uint32_t c = __ffs(b) - 1;
        s.x[nb][(size_t)k * P + c] = x0;
        s.msg[nb][(size_t)k * P + c] = m0;
      }
    }
  }
}

// The refilled slots' membership bits: block c sets bit c on its set's nodes.
__global__ void ppr_members_kernel(PprStream s) {
  const PprCtl* ctl = s.ctl;
  const uint32_t c = blockIdx.x;
  if (!((*(volatile const uint32_t*)&ctl->refilled >> c) & 1)) return;
  const uint32_t set = ctl->slot_set[c];
  for (uint64_t q = s.offsets[set] + threadIdx.x; q < s.offsets[set + 1]; q += blockDim.x)
    atomicOr(s.member + s.perm[s.nodes[q]], 1u << c);
}

// max_iter = 0: every set's ranks are the start vector.
__global__ void ppr_start_out_kernel(PprStream s) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < (uint64_t)s.width * s.n;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(q % s.n);
    s.ranks[q] = tomb_bit(s.tomb, s.perm[i]) ? 0.0 : s.start;
  }
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < s.width; q += gridDim.x * blockDim.x)
    s.iterations[q] = 0;
}

// Blocks of 8 warps (P = 8, 16) or kPull32Warps (P = 32), at most one warp a unit.
static uint32_t ppr_grid(const wc_version* v, uint32_t P, uint32_t blocks_per_sm) {
  const uint32_t warps = P == 32 ? kPull32Warps : 8;
  return std::max<uint32_t>(1, std::min<uint32_t>(max_blocks((int)blocks_per_sm),
                                                  (v->loc.csc.schedule.count + warps - 1) / warps));
}

// The run's scratch, acquired before anything is queued or captured.
static wc_status ppr_reserve(Ctx& ctx, uint32_t P, uint32_t blocks_per_sm) {
  wc_version* v = ctx.v;
  const uint64_t n = v->n;
  const uint32_t grid = ppr_grid(v, P, blocks_per_sm);
  DevBuf* b;
  WC_TRY(ctx.scratch(POOL_BATCH_0, n * P * 8 * 2, &b));
  WC_TRY(ctx.scratch(POOL_BATCH_1, n * P * 8 * 2, &b));
  WC_TRY(ctx.scratch(POOL_BATCH_2, n * 4, &b));
  WC_TRY(ctx.scratch(POOL_BATCH_3, 4096 + (uint64_t)grid * P * 16, &b));
  return ctx.scratch(POOL_BATCH_4,
                     (uint64_t)std::max<uint32_t>(v->loc.csc.schedule.slots, 1) * P *
                         sizeof(Partial<double, WC_OP_PLUS>), &b);
}

template <int P>
static void ppr_queue_iteration(Ctx& ctx, const PprStream& s, uint32_t grid, bool weighted,
                                Partial<double, WC_OP_PLUS>* carry) {
  wc_version* v = ctx.v;
  if constexpr (P == 32) {
    constexpr size_t smem32 = kPull32Smem;
    if (weighted)
      note_launch(), ppr_iter32_kernel<double><<<grid, kPull32Warps * 32, smem32, ctx.stream>>>(
          view_of<double>(v->loc.csc, v->loc.csc.weights.ptr), s, carry);
    else
      note_launch(), ppr_iter32_kernel<void><<<grid, kPull32Warps * 32, smem32, ctx.stream>>>(
          view_of<void>(v->loc.csc, nullptr), s, carry);
  } else {
    if (weighted)
      note_launch(), ppr_iter_kernel<P, double><<<grid, 256, 0, ctx.stream>>>(
          view_of<double>(v->loc.csc, v->loc.csc.weights.ptr), s, carry);
    else
      note_launch(), ppr_iter_kernel<P, void><<<grid, 256, 0, ctx.stream>>>(
          view_of<void>(v->loc.csc, nullptr), s, carry);
  }
  note_launch(), ppr_rows_kernel<P><<<max_blocks(4), 256, 0, ctx.stream>>>(s);
  note_launch(), ppr_members_kernel<<<P, 128, 0, ctx.stream>>>(s);
}

// Runs `width` sets through P slots.  `nodes`/`offsets`/`shares` are the
// sets in device memory; ranks (width × n) and iterations (width) are
// written in set order.
template <int P>
wc_status ppr_stream(Ctx& ctx, const PageRankRun& base, const uint64_t* nodes,
                     const uint64_t* offsets, const double* shares, uint32_t width, double* ranks,
                     uint32_t* iterations, uint32_t blocks_per_sm) {
  wc_version* v = ctx.v;
  const uint32_t n = (uint32_t)v->n;
  const uint32_t grid = ppr_grid(v, P, blocks_per_sm);
  WC_TRY(ppr_reserve(ctx, P, blocks_per_sm));
  DevBuf *xb, *mb, *memb, *sb, *cb;
  WC_TRY(ctx.scratch(POOL_BATCH_0, (uint64_t)n * P * 8 * 2, &xb));
  WC_TRY(ctx.scratch(POOL_BATCH_1, (uint64_t)n * P * 8 * 2, &mb));
  WC_TRY(ctx.scratch(POOL_BATCH_2, (uint64_t)n * 4, &memb));
  WC_TRY(ctx.scratch(POOL_BATCH_3, 4096 + (uint64_t)grid * P * 16, &sb));
  WC_TRY(ctx.scratch(POOL_BATCH_4,
                     (uint64_t)std::max<uint32_t>(v->loc.csc.schedule.slots, 1) * P *
                         sizeof(Partial<double, WC_OP_PLUS>), &cb));
  static_assert(sizeof(PprCtl) <= 4096, "the control block fits its page");
  PprStream s{};
  s.n = n;
  s.width = width;
  s.max_iter = base.opts.max_iter;
  s.x[0] = xb->as<double>();
  s.x[1] = s.x[0] + (size_t)n * P;
  s.msg[0] = mb->as<double>();
  s.msg[1] = s.msg[0] + (size_t)n * P;
  s.out = base.s.out;
  s.member = memb->as<uint32_t>();
  s.shares = shares;
  s.nodes = nodes;
  s.offsets = offsets;
  s.tomb = base.s.tomb;
  s.perm = v->loc.perm.as<uint32_t>();
  s.start = base.s.start;
  s.damping = base.s.damping;
  s.teleport = base.s.teleport;
  s.threshold = base.s.threshold;
  s.has_tol = base.s.has_tol;
  s.ctl = sb->as<PprCtl>();
  s.partials = reinterpret_cast<double*>(sb->as<unsigned char>() + 4096);
  s.ranks = ranks;
  s.iterations = iterations;
  s.err = v->error.as<DeviceError>();
  if (s.max_iter == 0) {
    note_launch(), ppr_start_out_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(s);
    return cuda_status(cudaGetLastError(), ctx.detail, "batched pagerank");
  }
  const bool weighted = base.opts.weighted != 0 && v->weighted;
  auto* carry = cb->as<Partial<double, WC_OP_PLUS>>();
  if constexpr (P == 32) {
    constexpr int smem32 = (int)kPull32Smem;
    WC_CUDA(cudaFuncSetAttribute(ppr_iter32_kernel<double>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem32), ctx.detail);
    WC_CUDA(cudaFuncSetAttribute(ppr_iter32_kernel<void>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem32), ctx.detail);
  }
  // Greedy hand-out over P slots: no slot runs longer than the mean load
  // plus one set, so this many global iterations always finish every set.
  const uint64_t bound = ((uint64_t)width * s.max_iter + P - 1) / P + s.max_iter;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool caller_capturing = cudaStreamIsCapturing(ctx.stream, &cs) == cudaSuccess &&
                                cs != cudaStreamCaptureStatusNone;
  s.pace = caller_capturing ? nullptr : v->pace_dev;
  WC_CUDA(cudaMemsetAsync(memb->ptr, 0, (uint64_t)n * 4, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(sb->ptr, 0, 4096, ctx.stream), ctx.detail);
  note_launch(), ppr_init_kernel<P><<<grid, 256, 0, ctx.stream>>>(s);
  note_launch(), ppr_members_kernel<<<P, 128, 0, ctx.stream>>>(s);
  if (caller_capturing) {
    // No progress can be read while the caller captures: every iteration
    // the bound allows is queued (those past the end return at once).
    for (uint64_t g = 0; g < bound; g++) ppr_queue_iteration<P>(ctx, s, grid, weighted, carry);
    return cuda_status(cudaGetLastError(), ctx.detail, "batched pagerank");
  }
  WC_CUDA(cudaGetLastError(), ctx.detail);
  cudaGraphExec_t chunk = nullptr;
  const std::string key = "ppr/" + std::to_string(P) + "/" + std::to_string(grid) + "/" +
                          std::to_string(weighted);
  const uint64_t before = g_launches.load();
  WC_TRY(ctx.capture(key, [&] {
    for (uint32_t q = 0; q < kChunkIterations; q++)
      ppr_queue_iteration<P>(ctx, s, grid, weighted, carry);
    return cuda_status(cudaGetLastError(), ctx.detail, "batched pagerank");
  }, &chunk));
  const uint64_t per_chunk = g_launches.load() - before;
  g_launches.fetch_sub(per_chunk);  // counted again at each replay
  // The progress words are the version's; earlier work on the stream that
  // reports in them must have ended before they are reset.
  WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
  volatile uint32_t* pace = v->pace_host;
  pace[0] = 0;
  pace[1] = 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (uint64_t g = 0; g < bound; g += kChunkIterations) {
    bool done = false;
    while (!(done = pace[1] != 0) && g >= (uint64_t)pace[0] + 2 * kChunkIterations) {
      if (ctx.cancelled() || cudaStreamQuery(ctx.stream) != cudaErrorNotReady) break;
      std::this_thread::yield();
    }
    if (done || ctx.cancelled()) break;
    const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                        std::chrono::steady_clock::now() - t0).count();
    if ((uint64_t)ms > ctx.timeout_ms) break;  // finish() reports the timeout
    WC_CUDA(cudaGraphLaunch(chunk, ctx.stream), ctx.detail);
    g_launches.fetch_add(per_chunk);
  }
  return WC_OK;
}

typedef wc_status (*PprFn)(Ctx&, const PageRankRun&, const uint64_t*, const uint64_t*,
                           const double*, uint32_t, double*, uint32_t*, uint32_t);

static PprFn ppr_for(uint32_t p) {
  switch (p) {
    case 8: return ppr_stream<8>;
    case 16: return ppr_stream<16>;
    default: return ppr_stream<32>;
  }
}

// Times the streaming run per slot count and blocks per SM on 64 one-node
// sets (10 iterations each) and keeps the fastest.
wc_status tune_ppr(Ctx& ctx, uint32_t width, wc_schedule* best) {
  wc_version* v = ctx.v;
  const uint32_t sample = std::max<uint32_t>(1, std::min<uint32_t>(width, 64));
  std::vector<uint64_t> nodes;
  sample_nodes((uint32_t)v->n, sample, nodes, 0x9e11u);
  std::vector<uint64_t> offs(sample + 1);
  for (uint32_t c = 0; c <= sample; c++) offs[c] = c;
  std::vector<double> shares(sample, 1.0);
  DevBuf *N, *F, *R, *I, *SH;
  WC_TRY(ctx.scratch(POOL_BATCH_11, sample * 8, &SH));
  WC_TRY(ctx.scratch(POOL_BATCH_5, sample * 8, &N));
  WC_TRY(ctx.scratch(POOL_BATCH_6, (sample + 1) * 8, &F));
  WC_TRY(ctx.scratch(POOL_BATCH_7, (uint64_t)sample * v->n * 8, &R));
  WC_TRY(ctx.scratch(POOL_BATCH_9, sample * 4, &I));
  WC_CUDA(cudaMemcpyAsync(SH->ptr, shares.data(), sample * 8, cudaMemcpyHostToDevice, ctx.stream),
          ctx.detail);
  WC_CUDA(cudaMemcpyAsync(N->ptr, nodes.data(), sample * 8, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemcpyAsync(F->ptr, offs.data(), (sample + 1) * 8, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
  wc_pagerank_opts o{0.85, 1e-10, 1, -1, 10, nullptr};
  PageRankRun base;
  WC_TRY(base.setup(ctx, &o, nullptr, nullptr, true));
  cudaEvent_t a, b;
  WC_CUDA(cudaEventCreate(&a), ctx.detail);
  WC_CUDA(cudaEventCreate(&b), ctx.detail);
  float best_ms = 1e30f;
  for (uint32_t P : {8u, 16u, 32u})
    for (uint32_t bps : {2u, 3u, 4u, 5u, 6u}) {
      // The 32-slot kernel's 4-warp blocks fit more an SM than the others'.
      if (P == 32 ? bps < 3 : bps > 4) continue;
      float ms = 0;
      for (int rep = 0; rep < 2; rep++) {
        WC_CUDA(cudaEventRecord(a, ctx.stream), ctx.detail);
        WC_TRY(ppr_for(P)(ctx, base, N->as<uint64_t>(), F->as<uint64_t>(), SH->as<double>(),
                          sample, R->as<double>(), I->as<uint32_t>(), bps));
        WC_CUDA(cudaEventRecord(b, ctx.stream), ctx.detail);
        WC_CUDA(cudaEventSynchronize(b), ctx.detail);
        WC_CUDA(cudaEventElapsedTime(&ms, a, b), ctx.detail);
      }
      if (ms < best_ms) {
        best_ms = ms;
        *best = wc_schedule{P, 1, bps, 0};
      }
    }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_ppr_batched(wc_version* v, const wc_call* call, const wc_pagerank_opts* o,
                         const uint64_t* seed_nodes, const uint64_t* seed_offsets, uint32_t width,
                         double* ranks_out, uint32_t* iterations_out) {
  if (!v || !o || (width && (!seed_offsets || !ranks_out))) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  if (width == 0) return WC_OK;
  const uint64_t n = v->n;
  std::vector<uint64_t> offs(width + 1);
  WC_CUDA(cudaMemcpy(offs.data(), seed_offsets, (width + 1) * 8, cudaMemcpyDefault), ctx.detail);
  std::vector<uint64_t> nodes(offs[width]);
  if (!nodes.empty())
    WC_CUDA(cudaMemcpy(nodes.data(), seed_nodes, nodes.size() * 8, cudaMemcpyDefault), ctx.detail);
  WC_TRY(ctx.begin());
  PageRankRun base;
  WC_TRY(base.setup(ctx, o, nullptr, nullptr, true));
  // Each set's personalisation (pagerank/mod.rs:155-199 with a seed of 1
  // on the set): the set's size summed in the reference's order is exact
  // (integers), then 1 / size, then 1 × that share.
  std::vector<double> shares(width);
  std::vector<uint64_t> dedup;
  for (uint32_t c = 0; c < width; c++) {
    dedup.assign(nodes.begin() + offs[c], nodes.begin() + offs[c + 1]);
    std::sort(dedup.begin(), dedup.end());
    dedup.erase(std::unique(dedup.begin(), dedup.end()), dedup.end());
    for (uint64_t q : dedup)
      if (q >= n) {
        if (ctx.detail) ctx.detail->node = q;
        return WC_NODE_OUTSIDE_ID_SPACE;
      }
    double total;
    WC_TRY((wc_status)sql_float<F_DIV>(1.0, (double)dedup.size(), &total));
    shares[c] = total;
  }
  Operand N(POOL_BATCH_5), F(POOL_BATCH_6), R(POOL_BATCH_7);
  WC_TRY(N.in(ctx, seed_nodes, std::max<uint64_t>(nodes.size(), 1) * 8));
  WC_TRY(F.in(ctx, seed_offsets, (width + 1) * 8));
  WC_TRY(R.output(ctx, ranks_out, (uint64_t)width * n * 8));
  DevBuf* its;
  WC_TRY(ctx.scratch(POOL_BATCH_9, (uint64_t)width * 4, &its));
  const auto key = ((uint64_t)WC_BATCH_PPR << 32) | width;
  const wc_schedule sched = v->tuned.count(key) ? v->tuned[key] : wc_schedule{32, 1, 5, 0};
  const uint32_t P = sched.columns_per_pass <= 8 ? 8 : sched.columns_per_pass <= 16 ? 16 : 32;
  const uint32_t bps = sched.blocks_per_sm ? sched.blocks_per_sm : 5;
  DevBuf* sh;
  WC_TRY(ctx.scratch(POOL_BATCH_11, (uint64_t)width * 8, &sh));
  WC_CUDA(cudaMemcpyAsync(sh->ptr, shares.data(), (uint64_t)width * 8, cudaMemcpyHostToDevice,
                          ctx.stream), ctx.detail);
  WC_TRY(ppr_for(P)(ctx, base, static_cast<const uint64_t*>(N.dev),
                    static_cast<const uint64_t*>(F.dev), sh->as<double>(), width,
                    static_cast<double*>(R.dev), its->as<uint32_t>(), bps));
  WC_TRY(R.out(ctx));
  if (iterations_out)
    WC_CUDA(cudaMemcpyAsync(iterations_out, its->ptr, width * 4, cudaMemcpyDefault, ctx.stream),
            ctx.detail);
  return locality_status(ctx, ctx.finish());
}

}  // extern "C"
