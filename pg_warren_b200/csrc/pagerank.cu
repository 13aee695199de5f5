// pagerank.cu — wc_pagerank: compute/pagerank/mod.rs:96-287 on the device.
//
// The reference runs, per iteration, `spread` (msg = x / out, the dangling
// rank summed), a plus_times pull over the reverse CSR, and `advance`
// (x ← d·(y + dangling·p) + (1−d)·p with the L1 change), each step's
// arithmetic as SQL float8 does it.  Here one kernel per iteration does all
// three: the pull of row i is followed at once by its advance and by the
// spread of the new x_i into the next iteration's message, so the messages
// are read once and x once per iteration.  The two sums (the L1 change and
// the next dangling rank) are reduced per block and then, by the last block
// to finish, in block order, so results do not vary from run to run.  That
// block also applies the stop test (delta < live × tol in SQL order) and
// raises a device flag on which later iterations return at once, so a
// call's iterations are queued without a round trip per iteration.
//
// Floating-point reassociation: rows of more than 256 entries, and the two
// sums, are added in another order than the reference's sequential folds
// (documented; the ranks stay within 1e-12 relative L1).  The seeded
// personalisation's sum is computed in the reference's own order (65536-
// element chunks folded sequentially, combined in order).
#include "operand.h"
#include "pagerank.h"
#include "pull.cuh"
#include "sqlfloat.cuh"
#include "upload.h"

namespace wc {

constexpr uint64_t kChunk = 1 << 16;  // compute/reduce.rs:20



__device__ inline bool tomb_at(const uint64_t* t, uint32_t i) {
  return t && ((t[i >> 6] >> (i & 63)) & 1);
}

// A fixed-order sum of two values over the block: lanes, then warps in
// order.  The result is in thread 0.
__device__ inline void block_sum_two(double& a, double& b) {
  __shared__ double sa[32], sb[32];
  const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  __syncthreads();
  if (lane == 0) {
    sa[wid] = a;
    sb[wid] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (unsigned w = 0; w < blockDim.x / 32; w++) {
      ta += sa[w];
      tb += sb[w];
    }
    a = ta;
    b = tb;
  }
}

// Sums two values per thread over the block, then over the blocks' sums
// in the last block to arrive (each of its threads folding a fixed stride
// of them, then the block in fixed order), so the totals do not depend on
// which block arrives last.  Returns true in thread 0 of that block, with
// the totals in a, b.
// `before`: block partials an earlier kernel of the same step stored at
// the front of `partials` (added in, first).
__device__ inline bool reduce_two(double& a, double& b, double* partials, unsigned* counter,
                                  unsigned before = 0) {
  __shared__ bool last;
  block_sum_two(a, b);
  if (threadIdx.x == 0) {
    partials[2 * (before + blockIdx.x)] = a;
    partials[2 * (before + blockIdx.x) + 1] = b;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double ta = 0.0, tb = 0.0;
  for (unsigned k = threadIdx.x; k < before + gridDim.x; k += blockDim.x) {
    ta += __ldcg(partials + 2 * k);
    tb += __ldcg(partials + 2 * k + 1);
  }
  block_sum_two(ta, tb);
  if (threadIdx.x != 0) return false;
  *counter = 0;
  a = ta;
  b = tb;
  return true;
}

// The reference's sum of a seed over live rows (reduce.rs:137-153, 266-279):
// each 65536-element chunk folded sequentially from +0.
// Block c sums chunk c of the live seed values in index order: warps 1..
// stage the next 2,048 terms in shared memory while thread 0 adds the
// current ones.  A tombstoned row's term is +0.0, which leaves a sum that
// starts at +0.0 unchanged, as skipping it does.
constexpr uint32_t kSeedStage = 2048;

__global__ void __launch_bounds__(256) seed_chunks_kernel(const double* seed, const uint64_t* tomb,
                                                          uint64_t n, double* partial) {
  __shared__ double stage[2][kSeedStage];
  const uint64_t c0 = (uint64_t)blockIdx.x * kChunk;
  const uint64_t c1 = min(n, c0 + kChunk);
  const uint32_t rounds = (uint32_t)((c1 - c0 + kSeedStage - 1) / kSeedStage);
  auto fill = [&](uint32_t r, uint32_t first) {
    double* st = stage[r & 1];
    for (uint32_t q = threadIdx.x - first; q < kSeedStage; q += blockDim.x - first) {
      const uint64_t i = c0 + (uint64_t)r * kSeedStage + q;
      st[q] = (i < c1 && !tomb_at(tomb, (uint32_t)i)) ? seed[i] : 0.0;
    }
  };
  double sum = 0.0;
  fill(0, 0);
  __syncthreads();
  for (uint32_t r = 0; r < rounds; r++) {
    if (threadIdx.x == 0) {
      const double* st = stage[r & 1];
#pragma unroll 16
      for (uint32_t q = 0; q < kSeedStage; q++) sum = sum + st[q];
    } else if (threadIdx.x >= 32 && r + 1 < rounds) {
      fill(r + 1, 32);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sum;
}

__global__ void seed_shares_kernel(const double* seed, const uint64_t* tomb, uint32_t n,
                                   const double* partial, uint32_t chunks, double* shares,
                                   DeviceError* err) {
  // total = 1 / (chunk sums added in chunk order); every thread recomputes
  // the short fold so no second launch is needed.
  double sum = 0.0;
  for (uint32_t c = 0; c < chunks; c++) sum = sum + partial[c];
  double total;
  int32_t s = sql_float<F_DIV>(1.0, sum, &total);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (s) {
      raise(err, s);
      return;
    }
    double share = 0.0;
    if (!tomb_at(tomb, i)) {
      int32_t e = sql_float<F_MUL>(seed[i], total, &share);
      if (e) raise(err, e, i);
    }
    shares[i] = share;
  }
}

// spread (mod.rs:204-232) for one row: the message, and the row's dangling
// rank (x where out is not above 0 in SQL order).
__device__ inline double spread_row(double x, double out, double* msg, DeviceError* err,
                                    uint32_t row) {
  if (sql_cmp_f(out, 0.0) > 0) {
    double m;
    int32_t s = sql_float<F_DIV>(x, out, &m);
    if (s) raise(err, s, row);
    *msg = m;
    return 0.0;
  }
  *msg = 0.0;
  return x;
}

__global__ void pr_init_kernel(PrState s) {
  double none = 0.0, dangling = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += gridDim.x * blockDim.x) {
    double x = tomb_at(s.tomb, i) ? 0.0 : s.start;
    s.x[0][i] = x;
    dangling += spread_row(x, s.out[i], &s.msg[0][i], s.err, i);
  }
  if (reduce_two(none, dangling, s.partials, s.counter)) {
    s.dangling[0] = dangling;
    *s.iterations = 0;
    *s.done = 0;
  }
}

// advance (mod.rs:245-282) and the next spread, for the row the pull ends.
struct PrEpi {
  const PrState* s;
  int cur;
  double dangling_in;
  double delta;
  double dangling_out;
  // The row's operands, requested before its pull so they arrive with it.
  struct Pre {
    double old, out, share;
    bool dead;
  };
  __device__ Pre pre(uint32_t i) const {
    const PrState& st = *s;
    Pre p;
    p.dead = tomb_at(st.tomb, i);
    p.share = st.shares ? st.shares[i] : st.start;
    p.old = st.x[cur][i];
    p.out = st.out[i];
    return p;
  }
  __device__ void row(uint32_t i, bool present, double y, const Pre& pr) {
    const PrState& st = *s;
    if (!present) y = 0.0;  // an empty row writes the plus identity
    double next = 0.0;
    if (!pr.dead) {
      const double p = pr.share;
      double dp, flowed, a, b;
      int32_t e = sql_float<F_MUL>(dangling_in, p, &dp);
      if (!e) e = sql_float<F_ADD>(y, dp, &flowed);
      if (!e) e = sql_float<F_MUL>(st.damping, flowed, &a);
      if (!e) e = sql_float<F_MUL>(st.teleport, p, &b);
      if (!e) e = sql_float<F_ADD>(a, b, &next);
      if (e) raise(st.err, e, i);
    }
    delta += fabs(next - pr.old);
    st.x[cur ^ 1][i] = next;
    dangling_out += spread_row(next, pr.out, &st.msg[cur ^ 1][i], st.err, i);
  }
};

// Unweighted, four blocks an SM (64 registers) keep more gathers in flight;
// with weights the extra registers would spill, so three.
// The step's close, by the last block of its last kernel: the stop test,
// the cancel word and the progress words.
__device__ inline void pr_close(const PrState& s, uint32_t it, double delta, double dangling) {
  s.delta[it] = delta;
  s.dangling[it + 1] = dangling;
  *s.iterations = it + 1;
  if (s.has_tol && sql_cmp_f(delta, s.threshold) < 0) *s.done = 1;
  // The caller's cancel word (host memory, mapped) is read once per
  // iteration, here; the next iteration then returns at once.
  if (*(volatile const int32_t*)s.cancel) {
    raise(s.err, WC_CANCELLED);
    *s.done = 1;
  }
  // Tell the host how far the solve is, so it stops queueing iterations.
  if (s.pace) {
    volatile uint32_t* pace = s.pace;
    pace[1] = *s.done;
    pace[0] = it + 1;
  }
}

// DEFER: the long rows' pieces only store their partials, and
// pr_long_kernel finishes those rows and the step; each block here leaves
// its sums at the front of the partials.
template <class W, bool SPLIT, bool DEFER>
__global__ void __launch_bounds__(kPullThreads, WSize<W>::v == 0 ? 4 : 3)
    pr_iter_kernel(CsrView<W> A, PrState s, uint32_t it) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (*(volatile int32_t*)s.done) return;
  const int cur = it & 1;
  PrEpi epi{&s, cur, s.dangling[it], 0.0, 0.0};
  PullRing<double, W>* ring = reinterpret_cast<PullRing<double, W>*>(smem) + (threadIdx.x >> 5);
  pull_units<double, WC_PLUS_TIMES, W, PrEpi, SPLIT, DEFER>(A, s.msg[cur], epi, s.err, ring);
  double delta = epi.delta, dangling = epi.dangling_out;
  if constexpr (DEFER) {
    block_sum_two(delta, dangling);
    if (threadIdx.x == 0) {
      s.partials[2 * blockIdx.x] = delta;
      s.partials[2 * blockIdx.x + 1] = dangling;
    }
    return;
  }
  if (reduce_two(delta, dangling, s.partials, s.counter)) pr_close(s, it, delta, dangling);
}

// The long rows of a step run with DEFER: a warp per row combines its
// pieces' partials in piece order (as the last piece to arrive does
// otherwise), then the row's advance and spread; the last block reduces
// both kernels' block sums in a fixed order and closes the step.
__global__ void __launch_bounds__(256)
    pr_long_kernel(const uint4* longs, uint32_t long_count,
                   const Partial<double, semiring_add(WC_PLUS_TIMES)>* carry, PrState s,
                   uint32_t it, uint32_t first_blocks) {
  if (*(volatile int32_t*)s.done) return;
  const int cur = it & 1;
  PrEpi epi{&s, cur, s.dangling[it], 0.0, 0.0};
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < long_count; r += warps) {
    const uint4 L = longs[r];  // row, first slot, pieces
    PrEpi::Pre pre{};
    if (lane == 0) pre = epi.pre(L.x);
    const auto total =
        combine_pieces<double, semiring_add(WC_PLUS_TIMES), 1>(carry, L.y, L.z, 0, lane);
    if (lane == 0) {
      double v;
      const int32_t st = total.acc.value(&v);
      if (st) raise(s.err, st, L.x);
      epi.row(L.x, true, v, pre);
    }
  }
  double delta = epi.delta, dangling = epi.dangling_out;
  if (reduce_two(delta, dangling, s.partials, s.counter, first_blocks))
    pr_close(s, it, delta, dangling);
}

template <class W, bool SPLIT, bool DEFER>
static wc_status set_iter_attributes(const PullLaunch& L) {
  constexpr size_t smem = pull_smem_bytes<double, W>();
  static const cudaError_t attr = cudaFuncSetAttribute(
      pr_iter_kernel<W, SPLIT, DEFER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cuda_status(attr, L.detail, "pagerank kernel attributes");
}

// One iteration: pr_iter_kernel over L's units, and with `longs` (the
// schedule's long rows, DEFER) pr_long_kernel after it on `long_grid` blocks.
template <class W>
wc_status launch_iter(const PullLaunch& L, const PrState& s, uint32_t it, uint32_t blocks,
                      const Schedule* longs = nullptr, uint32_t long_grid = 0) {
  CsrView<W> A{L.off, L.tgt, static_cast<const W*>(L.weights), L.units, L.unit_count, L.counters,
               L.carry, L.hot};
  constexpr size_t smem = pull_smem_bytes<double, W>();
  if (longs) {
    WC_TRY((set_iter_attributes<W, true, true>(L)));
    note_launch(), pr_iter_kernel<W, true, true><<<blocks, kPullThreads, smem, L.stream>>>(A, s, it);
    note_launch(), pr_long_kernel<<<long_grid, 256, 0, L.stream>>>(
        longs->long_list.as<uint4>(), longs->long_rows,
        static_cast<const Partial<double, semiring_add(WC_PLUS_TIMES)>*>(L.carry), s, it, blocks);
  } else if (L.hot) {
    WC_TRY((set_iter_attributes<W, true, false>(L)));
    note_launch(), pr_iter_kernel<W, true, false><<<blocks, kPullThreads, smem, L.stream>>>(A, s, it);
  } else {
    WC_TRY((set_iter_attributes<W, false, false>(L)));
    note_launch(), pr_iter_kernel<W, false, false><<<blocks, kPullThreads, smem, L.stream>>>(A, s, it);
  }
  return WC_OK;
}

wc_status prepare_pull(Ctx& ctx, DevCsr& csr, int semiring, int weighted_flag, int dtype,
                       uint32_t width, PullLaunch& L);
wc_status launch_pull(const PullLaunch& L, int dtype, const void* x, void* y);

wc_status launch_pr_init(const PrState& s, uint32_t grid, cudaStream_t stream) {
  note_launch(), pr_init_kernel<<<grid, kPullThreads, 0, stream>>>(s);
  return cuda_status(cudaGetLastError(), nullptr, "pagerank init");
}

wc_status launch_part_iteration(const PullLaunch& L, const PrState& s, uint32_t it,
                                uint32_t blocks) {
  if (L.weight_kind == WEIGHTS_F64) return launch_iter<double>(L, s, it, blocks);
  return launch_iter<void>(L, s, it, blocks);
}

uint64_t live_count(const uint64_t* tomb, uint64_t n) {
  uint64_t dead = 0;
  if (tomb)
    for (uint64_t w = 0; w < (n + 63) / 64; w++) {
      uint64_t word = tomb[w];
      if (w == n / 64 && (n & 63)) word &= (1ull << (n & 63)) - 1;
      dead += __builtin_popcountll(word);
    }
  return n - dead;
}

uint32_t pagerank_long_grid(const DevCsr& csc) {
  return std::max<uint32_t>(1, std::min<uint32_t>((csc.schedule.long_rows + 7) / 8, max_blocks(2)));
}

uint32_t pagerank_partial_blocks(const DevCsr& csc) {
  return pagerank_grid(csc) + pagerank_long_grid(csc);
}

uint32_t pagerank_grid(const DevCsr& csc) {
  return std::max<uint32_t>(1, std::min<uint32_t>((csc.schedule.count + kPullWarps - 1) / kPullWarps,
                                                  max_blocks(8)));
}

wc_status PageRankRun::setup(Ctx& ctx, const wc_pagerank_opts* o, const uint64_t* tomb_host,
                             const double* seed, bool in_locality_order) {
  wc_version* v = ctx.v;
  const uint64_t n = v->n;
  const uint64_t words = (n + 63) / 64;
  opts = *o;
  local = in_locality_order;
  // Tombstones: the caller's words, on the device.
  std::vector<uint64_t> host_words;
  const uint64_t* th = tomb_host;
  if (tomb_host && is_device_pointer(tomb_host)) {
    host_words.resize(words);
    WC_CUDA(cudaMemcpy(host_words.data(), tomb_host, words * 8, cudaMemcpyDeviceToHost),
            ctx.detail);
    th = host_words.data();
  }
  live = live_count(th, n);
  nodes = (double)live;
  double start;
  WC_TRY((wc_status)sql_float<F_DIV>(1.0, nodes, &start));
  double teleport;
  WC_TRY((wc_status)sql_float<F_SUB>(1.0, o->damping, &teleport));
  double threshold = 0.0;
  if (o->has_tol && o->max_iter > 0) WC_TRY((wc_status)sql_float<F_MUL>(nodes, o->tol, &threshold));
  const uint32_t blocks = pagerank_grid(csc(v));
  grid = blocks;
  long_grid = pagerank_long_grid(csc(v));
  const uint32_t partial_blocks = blocks + long_grid;
  WC_TRY(ctx.scratch(POOL_PR_X, 2 * n * 8, &x));
  WC_TRY(ctx.scratch(POOL_PR_MSG, 2 * n * 8, &msg));
  WC_TRY(ctx.scratch(POOL_PR_OUT, n * 8, &out));
  const uint64_t scalar_bytes = (2 * (uint64_t)o->max_iter + 8) * 8 + 2 * partial_blocks * 8 + 64;
  WC_TRY(ctx.scratch(POOL_PR_SCALARS, scalar_bytes, &scalars));
  uint64_t* tomb_dev = nullptr;
  if (th) {
    // In locality order the words are renumbered into the buffer's second half.
    WC_TRY(ctx.scratch(POOL_PR_TOMB, words * 8 * (local ? 2 : 1), &tomb));
    WC_CUDA(cudaMemcpyAsync(tomb->ptr, th, words * 8, cudaMemcpyHostToDevice, ctx.stream),
            ctx.detail);
    tomb_dev = tomb->as<uint64_t>();
    if (local) {
      WC_TRY(bits_to_locality(v, ctx.stream, tomb_dev, tomb_dev + words));
      tomb_dev += words;
    }
  }
  WC_CUDA(cudaMemsetAsync(scalars->ptr, 0, scalar_bytes, ctx.stream), ctx.detail);
  double* sc = scalars->as<double>();
  s = PrState{};
  s.n = (uint32_t)n;
  s.x[0] = x->as<double>();
  s.x[1] = x->as<double>() + n;
  s.msg[0] = msg->as<double>();
  s.msg[1] = msg->as<double>() + n;
  s.out = out->as<double>();
  s.tomb = tomb_dev;
  s.start = start;
  s.damping = o->damping;
  s.teleport = teleport;
  s.threshold = threshold;
  s.has_tol = o->has_tol != 0;
  s.delta = sc;
  s.dangling = sc + o->max_iter;
  s.partials = sc + 2 * (uint64_t)o->max_iter + 8;
  unsigned char* tail = reinterpret_cast<unsigned char*>(s.partials + 2 * partial_blocks);
  s.counter = reinterpret_cast<unsigned*>(tail);
  s.iterations = reinterpret_cast<uint32_t*>(tail + 8);
  s.done = reinterpret_cast<int32_t*>(tail + 16);
  s.cancel = v->cancel_dev;
  s.pace = v->pace_dev;
  s.err = v->error.as<DeviceError>();
  // out = plus_first over the forward CSR: each row's out-weight (in
  // locality order: into the second message buffer, then renumbered).
  PullLaunch L;
  WC_TRY(prepare_pull(ctx, v->fwd, WC_PLUS_FIRST, o->weighted, WC_F64, 1, L));
  WC_TRY(launch_pull(L, WC_F64, s.x[0], local ? s.msg[1] : out->ptr));
  if (local) WC_TRY(to_locality(v, ctx.stream, s.msg[1], out->as<double>()));
  // The personalisation, summed in dense-id order (the reference's chunks).
  if (seed) {
    Operand S(POOL_SEED);
    WC_TRY(S.in(ctx, seed, n * 8));
    const double* sd = static_cast<const double*>(S.dev);
    const uint32_t chunks = (uint32_t)((n + kChunk - 1) / kChunk);
    WC_TRY(ctx.scratch(POOL_PR_SHARES, n * 8 * (local ? 2 : 1) + (uint64_t)chunks * 8, &shares));
    double* partial = shares->as<double>() + n * (local ? 2 : 1);
    const uint64_t* tomb_ids = th ? tomb->as<uint64_t>() : nullptr;  // dense-id order
    if (chunks)
      note_launch(), seed_chunks_kernel<<<chunks, 256, 0, ctx.stream>>>(sd, tomb_ids, n, partial);
    note_launch(), seed_shares_kernel<<<max_blocks(4), 256, 0, ctx.stream>>>(sd, tomb_ids, (uint32_t)n, partial,
                                                             chunks, shares->as<double>(), s.err);
    s.shares = shares->as<double>();
    if (local) {
      WC_TRY(to_locality(v, ctx.stream, shares->as<double>(), shares->as<double>() + n));
      s.shares = shares->as<double>() + n;
    }
  }
  return cuda_status(cudaGetLastError(), ctx.detail, "pagerank setup");
}

wc_status PageRankRun::run(Ctx& ctx) {
  wc_version* v = ctx.v;
  WC_TRY(launch_pr_init(s, grid, ctx.stream));
  PullLaunch L;
  WC_TRY(prepare_pull(ctx, const_cast<DevCsr&>(csc(v)), WC_PLUS_TIMES, opts.weighted, WC_F64, 1, L));
  if (local) L.hot = kPageRankHotNodes;
  // With a tolerance the solve usually stops well before max_iter: the
  // host keeps at most kAhead iterations queued beyond the last one the
  // device reported, and stops queueing once the device reports the stop,
  // so few launches return at once on the done flag.
  constexpr uint32_t kAhead = 3;
  volatile uint32_t* pace = s.pace ? v->pace_host : nullptr;
  if (pace) {
    pace[0] = 0;
    pace[1] = 0;
  }
  ctx.phase_begin("iteration");
  for (uint32_t it = 0; it < opts.max_iter; it++) {
    // A cancel stops the queueing (the kernels queued read the device's
    // copy of the word, which finish() raises).
    if (ctx.cancelled()) break;
    if (pace && s.has_tol) {
      bool stop = false;
      while (!(stop = pace[1] != 0) && it >= pace[0] + kAhead) {
        if (ctx.cancelled() || cudaStreamQuery(ctx.stream) != cudaErrorNotReady) break;
        std::this_thread::yield();
      }
      if (stop) break;
    }
    // In the locality order the long rows are finished by a pass of their
    // own, after their pieces (no release/acquire arrival per piece).
    const Schedule* longs = local ? &csc(v).schedule : nullptr;
    if (L.weight_kind == WEIGHTS_F64) WC_TRY(launch_iter<double>(L, s, it, grid, longs, long_grid));
    else WC_TRY(launch_iter<void>(L, s, it, grid, longs, long_grid));
  }
  ctx.phase_end();
  return cuda_status(cudaGetLastError(), ctx.detail, "pagerank iterations");
}

wc_status PageRankRun::result(Ctx& ctx, double* ranks_dev_or_host, uint32_t* iterations_out,
                              double* margin) {
  uint32_t its = 0;
  WC_CUDA(cudaMemcpy(&its, s.iterations, 4, cudaMemcpyDeviceToHost), ctx.detail);
  if (opts.max_iter == 0) its = 0;
  const double* final_x = s.x[its & 1];
  if (local) {
    // Back to dense-id order, through the other rank buffer (free now).
    WC_TRY(from_locality(ctx.v, ctx.stream, final_x, s.x[(its & 1) ^ 1]));
    final_x = s.x[(its & 1) ^ 1];
  }
  WC_CUDA(cudaMemcpyAsync(ranks_dev_or_host, final_x, ctx.v->n * 8, cudaMemcpyDefault, ctx.stream),
          ctx.detail);
  WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
  if (iterations_out) *iterations_out = its;
  if (margin && its > 0) {
    double delta = 0.0;
    WC_CUDA(cudaMemcpy(&delta, s.delta + (its - 1), 8, cudaMemcpyDeviceToHost), ctx.detail);
    *margin = s.threshold != 0.0 ? delta / s.threshold : 0.0;
  }
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_pagerank(wc_version* v, const wc_call* call, const wc_pagerank_opts* o,
                      const uint64_t* tombstones, double* ranks, uint32_t* iterations) {
  if (!v || !o || !ranks) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  PageRankRun run;
  ctx.phase_begin("setup");
  WC_TRY(run.setup(ctx, o, tombstones, o->seed, true));
  ctx.phase_end();
  ctx.progress("iterating", 0, o->max_iter);
  WC_TRY(run.run(ctx));
  WC_TRY(locality_status(ctx, ctx.finish()));
  double margin = 0.0;
  WC_TRY(run.result(ctx, ranks, iterations, &margin));
  v->last_margin = margin;
  ctx.progress("iterating", iterations ? *iterations : 0, o->max_iter);
  return WC_OK;
}

double wc_pagerank_last_margin(const wc_version* v) { return v ? v->last_margin : 0.0; }

}  // extern "C"
