// batched_multi.cu — wc_minplus_batched: many min-plus searches run as one
// SpMM over P columns at a time (pull_multi.cuh), with every column
// stopping at its own iterate.  No reference counterpart; each column
// computes what compute_sql/library/sssp_vector.sql:14-66 computes over i64
// for its source alone — next starts as a copy of x, spmv(x → next,
// min_plus, transpose, accumulate min), stop when no distance fell or after
// max_iter iterations.  Versions whose distances fit 32 bits take the
// 32-bit path (batched_minplus32.cu).
// Each pass's iterations are queued without a host round trip: a control
// step after each iteration updates the columns still running on the
// device, and iterations with no column left return at once.
#include <algorithm>
#include <string>

#include "batched.h"
#include "operand.h"
#include "pagerank.h"
#include "columns.cuh"
#include "pull_multi.cuh"
#include "sqlfloat.cuh"

namespace wc {

// =================================================================== min-plus

struct MpState {
  uint32_t n;
  int64_t* x[2];            // n × P
  const uint32_t* caps;     // P (this pass)
  uint32_t k;               // columns in use
  uint32_t* running;        // bit per column
  uint32_t* fell;           // bit per column, this iteration
  uint32_t* executed;       // iterations run by any column
  uint32_t* iterations;     // the call's, indexed by cols[c]
  const uint32_t* cols;     // P: the call's column of each pass column
  DeviceError* err;
};

template <int P> struct MpEpi {
  const MpState* s;
  int cur;
  uint32_t run_bits;
  uint32_t fell_bits;
  __device__ void cell(uint32_t i, uint32_t c, bool present, int64_t t) {
    const int64_t old = s->x[cur][(size_t)i * P + c];
    int64_t next = old;
    if ((run_bits >> c) & 1 && present) next = t < old ? t : old;  // accumulate min
    if (next < old) fell_bits |= 1u << c;
    s->x[cur ^ 1][(size_t)i * P + c] = next;
  }
};

template <int P>
__global__ void mp_seed_kernel(MpState s, const uint64_t* sources) {
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < (size_t)s.n * P;
       x += (size_t)gridDim.x * blockDim.x)
    s.x[0][x] = INT64_MAX;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint32_t run = 0;
    for (uint32_t c = 0; c < s.k; c++) {
      s.iterations[s.cols[c]] = 0;
      if (s.caps[c] > 0) run |= 1u << c;
    }
    *s.running = run;
    *s.fell = 0;
    *s.executed = 0;
  }
}

template <int P>
__global__ void mp_sources_kernel(MpState s, const uint64_t* sources) {
  const uint32_t c = threadIdx.x;
  if (c < s.k) s.x[0][(size_t)sources[c] * P + c] = 0;
}

template <int P, class W>
__global__ void __launch_bounds__(256) mp_iter_kernel(CsrView<W> A, MpState s, uint32_t it,
                                                      Partial<int64_t, WC_OP_MIN>* carry) {
  const uint32_t run = *(volatile uint32_t*)s.running;
  if (!run) return;
  MpEpi<P> epi{&s, (int)(it & 1), run, 0};
  pull_multi<int64_t, WC_MIN_PLUS, W, P>(A, s.x[it & 1], epi, s.err, carry);
  unsigned bits = epi.fell_bits;
  for (int o = 16; o > 0; o >>= 1) bits |= __shfl_xor_sync(0xffffffffu, bits, o);
  if ((threadIdx.x & 31) == 0 && bits) atomicOr(s.fell, bits);
}

// After iteration `it` (0-based): a running column whose distances did not
// fall stops with it + 1 iterations; one at its cap stops too.  Columns that
// stopped keep their values (the next iteration copies them forward).
__global__ void mp_control_kernel(MpState s, uint32_t it) {
  if (threadIdx.x != 0) return;
  uint32_t run = *s.running, fell = *s.fell;
  if (run) *s.executed = it + 1;
  for (uint32_t c = 0; c < s.k; c++) {
    if (!((run >> c) & 1)) continue;
    s.iterations[s.cols[c]] = it + 1;
    if (!((fell >> c) & 1) || it + 1 >= s.caps[c]) run &= ~(1u << c);
  }
  *s.running = run;
  *s.fell = 0;
}

// out[cols[c] * n + i] (cols NULL: c) = x[i * P + c] from the buffer the
// last iteration wrote: a 32-node tile through shared memory.
template <int P, class T>
__global__ void columns_out_kernel(const T* x0, const T* x1, const uint32_t* executed, uint32_t n,
                                   uint32_t k, T* out, const uint32_t* cols) {
  __shared__ T tile[32][P + 1];
  const T* x = (*executed & 1) ? x1 : x0;
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
      if (i0 + r < n) out[(size_t)(cols ? cols[c] : c) * n + i0 + r] = tile[r][c];
    }
    __syncthreads();
  }
}

struct MpPass {
  DevBuf *x, *state, *carry;
};

template <int P>
wc_status mp_pass(Ctx& ctx, const uint64_t* sources, const uint32_t* caps_dev, const uint32_t* cols,
                  uint32_t k, uint32_t max_cap, int64_t* out, uint32_t* iterations_dev,
                  uint32_t blocks_per_sm) {
  wc_version* v = ctx.v;
  const uint32_t n = (uint32_t)v->n;
  DevBuf *xb, *stb, *cb;
  WC_TRY(ctx.scratch(POOL_BATCH_0, (uint64_t)n * P * 8 * 2, &xb));
  WC_TRY(ctx.scratch(POOL_BATCH_1, 128, &stb));
  WC_TRY(ctx.scratch(POOL_BATCH_2,
                     (uint64_t)std::max<uint32_t>(v->rev.schedule.slots, 1) * P *
                         sizeof(Partial<int64_t, WC_OP_MIN>), &cb));
  MpState s;
  s.n = n;
  s.x[0] = xb->as<int64_t>();
  s.x[1] = s.x[0] + (size_t)n * P;
  s.caps = caps_dev;
  s.k = k;
  s.running = stb->as<uint32_t>();
  s.fell = s.running + 1;
  s.executed = s.running + 2;
  s.iterations = iterations_dev;
  s.cols = cols;
  s.err = v->error.as<DeviceError>();
  note_launch(), mp_seed_kernel<P><<<max_blocks(4), 256, 0, ctx.stream>>>(s, sources);
  note_launch(), mp_sources_kernel<P><<<1, 32, 0, ctx.stream>>>(s, sources);
  const bool weighted = v->weighted;
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(
      max_blocks((int)blocks_per_sm), (v->rev.schedule.count + 7) / 8));
  auto* carry = cb->as<Partial<int64_t, WC_OP_MIN>>();
  for (uint32_t it = 0; it < max_cap; it++) {
    if (weighted && v->integral)
      note_launch(), mp_iter_kernel<P, int32_t><<<grid, 256, 0, ctx.stream>>>(
          view_of<int32_t>(v->rev, v->rev.iweights.ptr), s, it, carry);
    else if (weighted)
      note_launch(), mp_iter_kernel<P, double><<<grid, 256, 0, ctx.stream>>>(
          view_of<double>(v->rev, v->rev.weights.ptr), s, it, carry);
    else
      note_launch(), mp_iter_kernel<P, void><<<grid, 256, 0, ctx.stream>>>(view_of<void>(v->rev, nullptr), s, it,
                                                            carry);
    note_launch(), mp_control_kernel<<<1, 32, 0, ctx.stream>>>(s, it);
  }
  note_launch(), columns_out_kernel<P, int64_t><<<max_blocks(4), 256, 0, ctx.stream>>>(
      s.x[0], s.x[1], s.executed, n, k, out, cols);
  return cuda_status(cudaGetLastError(), ctx.detail, "batched min-plus pass");
}

// The pass's scratch, acquired before a pass is captured (a capture may
// not allocate); mp_pass then finds it in the pool.
static wc_status mp_reserve(Ctx& ctx, uint32_t P) {
  wc_version* v = ctx.v;
  DevBuf* b;
  WC_TRY(ctx.scratch(POOL_BATCH_0, (uint64_t)v->n * P * 8 * 2, &b));
  WC_TRY(ctx.scratch(POOL_BATCH_1, 128, &b));
  return ctx.scratch(POOL_BATCH_2,
                     (uint64_t)std::max<uint32_t>(v->rev.schedule.slots, 1) * P *
                         sizeof(Partial<int64_t, WC_OP_MIN>), &b);
}

typedef wc_status (*MpFn)(Ctx&, const uint64_t*, const uint32_t*, const uint32_t*, uint32_t,
                          uint32_t, int64_t*, uint32_t*, uint32_t);

static MpFn mp_for(uint32_t p) {
  switch (p) {
    case 1: return mp_pass<1>;
    case 2: return mp_pass<2>;
    case 4: return mp_pass<4>;
    case 8: return mp_pass<8>;
    case 16: return mp_pass<16>;
    default: return mp_pass<32>;
  }
}

// Seeded sample columns for the tuners.
void sample_nodes(uint32_t n, uint32_t count, std::vector<uint64_t>& out, uint64_t salt) {
  out.resize(count);
  uint64_t z = salt;
  for (uint32_t s = 0; s < count; s++) {
    z = z * 6364136223846793005ull + 1442695040888963407ull;
    out[s] = (z >> 17) % n;
  }
}

// Times one pass per candidate pass width on a sample of columns and keeps
// the fastest per column.
wc_status tune_minplus(Ctx& ctx, uint32_t width, wc_schedule* best) {
  wc_version* v = ctx.v;
  const uint32_t sample = std::min<uint32_t>(width, 64);
  std::vector<uint64_t> src;
  sample_nodes((uint32_t)v->n, sample, src, 0x5eedu);
  std::vector<uint32_t> caps(sample, 16), cols(sample);
  for (uint32_t c = 0; c < sample; c++) cols[c] = c;
  DevBuf *S, *C, *D, *I, *ident;
  WC_TRY(ctx.scratch(POOL_BATCH_5, sample * 8, &S));
  WC_TRY(ctx.scratch(POOL_BATCH_6, sample * 4, &C));
  WC_TRY(ctx.scratch(POOL_BATCH_7, (uint64_t)sample * v->n * 8, &D));
  WC_TRY(ctx.scratch(POOL_BATCH_9, sample * 4, &I));
  WC_TRY(ctx.scratch(POOL_BATCH_10, sample * 4, &ident));
  WC_CUDA(cudaMemcpyAsync(S->ptr, src.data(), sample * 8, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemcpyAsync(C->ptr, caps.data(), sample * 4, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemcpyAsync(ident->ptr, cols.data(), sample * 4, cudaMemcpyHostToDevice, ctx.stream),
          ctx.detail);
  cudaEvent_t a, b;
  WC_CUDA(cudaEventCreate(&a), ctx.detail);
  WC_CUDA(cudaEventCreate(&b), ctx.detail);
  float best_per = 1e30f;
  for (uint32_t P : {4u, 8u, 16u, 32u})
    for (uint32_t bps : {4u, 8u}) {
      if (P > sample && P != 4) continue;
      const uint32_t k = std::min(P, sample);
      float ms = 0;
      for (int rep = 0; rep < 2; rep++) {
        WC_CUDA(cudaEventRecord(a, ctx.stream), ctx.detail);
        WC_TRY(mp_for(P)(ctx, S->as<uint64_t>(), C->as<uint32_t>(), ident->as<uint32_t>(), k, 16,
                         D->as<int64_t>(), I->as<uint32_t>(), bps));
        WC_CUDA(cudaEventRecord(b, ctx.stream), ctx.detail);
        WC_CUDA(cudaEventSynchronize(b), ctx.detail);
        WC_CUDA(cudaEventElapsedTime(&ms, a, b), ctx.detail);
      }
      if (ms / k < best_per) {
        best_per = ms / k;
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

wc_status wc_minplus_batched(wc_version* v, const wc_call* call, const uint64_t* sources,
                             const uint32_t* max_hops, uint32_t width, int64_t* dist_out,
                             uint32_t* iterations_out) {
  if (!v || (width && (!sources || !max_hops || !dist_out))) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  if (width == 0) return WC_OK;
  std::vector<uint64_t> src(width);
  std::vector<uint32_t> caps(width);
  WC_CUDA(cudaMemcpy(src.data(), sources, width * 8, cudaMemcpyDefault), ctx.detail);
  WC_CUDA(cudaMemcpy(caps.data(), max_hops, width * 4, cudaMemcpyDefault), ctx.detail);
  for (uint64_t s : src)
    if (s >= v->n) {
      if (ctx.detail) ctx.detail->node = s;
      return WC_NODE_OUTSIDE_ID_SPACE;
    }
  WC_TRY(ctx.begin());
  // Passes take the searches in order of their caps, so that a pass's
  // columns stop at about the same iteration; results go back to each
  // search's own column.
  std::vector<uint32_t> order(width);
  for (uint32_t c = 0; c < width; c++) order[c] = c;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t p, uint32_t q) { return caps[p] < caps[q]; });
  std::vector<uint64_t> psrc(width);
  std::vector<uint32_t> pcaps(width);
  for (uint32_t c = 0; c < width; c++) {
    psrc[c] = src[order[c]];
    pcaps[c] = caps[order[c]];
  }
  DevBuf* pb;
  WC_TRY(ctx.scratch(POOL_BATCH_10, (uint64_t)width * 16, &pb));
  uint64_t* psrc_dev = pb->as<uint64_t>();
  uint32_t* pcaps_dev = reinterpret_cast<uint32_t*>(psrc_dev + width);
  uint32_t* pcols_dev = pcaps_dev + width;
  WC_CUDA(cudaMemcpyAsync(psrc_dev, psrc.data(), width * 8, cudaMemcpyHostToDevice, ctx.stream),
          ctx.detail);
  WC_CUDA(cudaMemcpyAsync(pcaps_dev, pcaps.data(), width * 4, cudaMemcpyHostToDevice, ctx.stream),
          ctx.detail);
  WC_CUDA(cudaMemcpyAsync(pcols_dev, order.data(), width * 4, cudaMemcpyHostToDevice, ctx.stream),
          ctx.detail);
  Operand D(POOL_BATCH_7), I(POOL_BATCH_8);
  WC_TRY(D.output(ctx, dist_out, (uint64_t)width * v->n * 8));
  DevBuf* its;
  WC_TRY(ctx.scratch(POOL_BATCH_9, (uint64_t)width * 4, &its));
  const auto key = ((uint64_t)WC_BATCH_MINPLUS << 32) | width;
  const wc_schedule sched = v->tuned.count(key) ? v->tuned[key] : wc_schedule{32, 1, 4, 0};
  const uint32_t P = std::max<uint32_t>(1, std::min<uint32_t>(32, sched.columns_per_pass));
  const uint32_t bps = sched.blocks_per_sm ? sched.blocks_per_sm : 4;
  // 32-bit distances when no value can leave the 32-bit range.
  const uint32_t cap_max = *std::max_element(caps.begin(), caps.end());
  if (v->max_abs_iweight >= 0 && (uint64_t)cap_max * (uint64_t)v->max_abs_iweight < (1ull << 30)) {
    const uint32_t P32 = width > 32 ? 64 : 32;
    WC_TRY(mp32_reserve(ctx, P32));
    for (uint32_t c0 = 0; c0 < width; c0 += P32) {
      const uint32_t k = std::min(P32, width - c0);
      uint32_t max_cap = 0;
      for (uint32_t c = c0; c < c0 + k; c++) max_cap = std::max(max_cap, pcaps[c]);
      const std::string gk = "minplus32/" + std::to_string(P32) + "/" + std::to_string(k) + "/" +
                             std::to_string(max_cap);
      WC_TRY(ctx.run_captured(gk, [&] {
        return mp32_for(P32)(ctx, psrc_dev + c0, pcaps_dev + c0, pcols_dev + c0, k, max_cap,
                             static_cast<int64_t*>(D.dev), its->as<uint32_t>(),
                             P32 == 64 ? 2 : 3);
      }));
    }
    WC_TRY(D.out(ctx));
    if (iterations_out)
      WC_CUDA(cudaMemcpyAsync(iterations_out, its->ptr, width * 4, cudaMemcpyDefault, ctx.stream),
              ctx.detail);
    return ctx.finish();
  }
  WC_TRY(mp_reserve(ctx, P));
  for (uint32_t c0 = 0; c0 < width; c0 += P) {
    const uint32_t k = std::min(P, width - c0);
    uint32_t max_cap = 0;
    for (uint32_t c = c0; c < c0 + k; c++) max_cap = std::max(max_cap, pcaps[c]);
    const std::string gk = "minplus/" + std::to_string(P) + "/" + std::to_string(k) + "/" +
                           std::to_string(max_cap) + "/" + std::to_string(bps);
    WC_TRY(ctx.run_captured(gk, [&] {
      return mp_for(P)(ctx, psrc_dev + c0, pcaps_dev + c0, pcols_dev + c0, k, max_cap,
                       static_cast<int64_t*>(D.dev), its->as<uint32_t>(), bps);
    }));
  }
  WC_TRY(D.out(ctx));
  if (iterations_out)
    WC_CUDA(cudaMemcpyAsync(iterations_out, its->ptr, width * 4, cudaMemcpyDefault, ctx.stream),
            ctx.detail);
  return ctx.finish();
}

}  // extern "C"
