// noalloc.cu — wc_pagerank_noalloc: PageRank whose per-call working memory
// is a fixed array in the module's global memory, so that a call allocates
// nothing on the device or the host.  The kernels are wc_pagerank's own
// (PageRankRun::run); only where the rank, message, out-weight, tombstone and
// stop-test buffers live differs.
//
// Who needs it: a caller that must not allocate while it serves a query — a
// database backend whose device memory is held by another allocator (a
// caching allocator that has reserved the rest of HBM), or one on a latency
// budget for which cudaMalloc/cudaFree, which may synchronise the device,
// are not acceptable.  The array is reserved when the module loads on a
// device and is never charged to a wc_budget.
#include <mutex>

#include "operand.h"
#include "pagerank.h"
#include "pull.cuh"
#include "sqlfloat.cuh"
#include "upload.h"

namespace wc {

wc_status prepare_pull(Ctx& ctx, DevCsr& csr, int semiring, int weighted_flag, int dtype,
                       uint32_t width, PullLaunch& L);
wc_status launch_pull(const PullLaunch& L, int dtype, const void* x, void* y);

// The per-call working memory: 2n + 2n + n doubles (ranks, messages,
// out-weights), the tombstone words, and the stop-test scalars.  64 MiB holds
// a graph of about 1.67 million nodes at the default 100 iterations.
constexpr uint64_t kStaticScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_pagerank_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
// The array's device address on each device, found once (the first call on
// that device) with the device current.
static void* g_scratch_addr[kMaxDevices];
// One caller at a time per device: every call on a device shares its array.
static std::mutex g_scratch_mu[kMaxDevices];

static uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

// The bytes a solve of n nodes and max_iter iterations needs, in the order
// they are laid out: x[2], msg[2], out, tombstones (if any: the caller's
// words and their renumbering into the locality order), scalars.
static uint64_t static_bytes(uint64_t n, uint32_t max_iter, uint32_t blocks, bool tomb) {
  uint64_t b = align256(2 * n * 8) * 2 + align256(n * 8);
  if (tomb) b += align256(2 * ((n + 63) / 64) * 8);
  b += align256((2 * (uint64_t)max_iter + 8) * 8 + 2 * (uint64_t)blocks * 8 + 64);
  return b;
}

// Counts the live rows of tombstones held in device memory, through a
// buffer on the stack.
static wc_status device_live_count(const uint64_t* tomb_dev, uint64_t n, uint64_t* live,
                                   wc_error_detail* detail) {
  uint64_t words[512];
  const uint64_t total = (n + 63) / 64;
  uint64_t dead = 0;
  for (uint64_t w0 = 0; w0 < total; w0 += 512) {
    const uint64_t k = std::min<uint64_t>(512, total - w0);
    WC_CUDA(cudaMemcpy(words, tomb_dev + w0, k * 8, cudaMemcpyDeviceToHost), detail);
    for (uint64_t q = 0; q < k; q++) {
      uint64_t word = words[q];
      if (w0 + q == n / 64 && (n & 63)) word &= (1ull << (n & 63)) - 1;
      dead += __builtin_popcountll(word);
    }
  }
  *live = n - dead;
  return WC_OK;
}

// PageRankRun::setup with the working memory carved from `base` instead of
// the version's scratch pool.  Everything the kernels read as a running
// total (deltas, dangling sums, block partials, the arrival counter, the
// iteration count, the done flag) is cleared here on every call; the rank
// and message vectors are written by pr_init_kernel before they are read.
static wc_status static_setup(Ctx& ctx, PageRankRun& run, const wc_pagerank_opts* o,
                              const uint64_t* tomb_in, unsigned char* base) {
  wc_version* v = ctx.v;
  const uint64_t n = v->n;
  run.opts = *o;
  const bool tomb_dev = tomb_in && is_device_pointer(tomb_in);
  if (tomb_dev) WC_TRY(device_live_count(tomb_in, n, &run.live, ctx.detail));
  else run.live = live_count(tomb_in, n);
  run.nodes = (double)run.live;
  double start, teleport, threshold = 0.0;
  WC_TRY((wc_status)sql_float<F_DIV>(1.0, run.nodes, &start));
  WC_TRY((wc_status)sql_float<F_SUB>(1.0, o->damping, &teleport));
  if (o->has_tol && o->max_iter > 0)
    WC_TRY((wc_status)sql_float<F_MUL>(run.nodes, o->tol, &threshold));
  run.local = true;  // wc_pagerank's own numbering, so the results are its
  run.grid = pagerank_grid(run.csc(v));
  run.long_grid = pagerank_long_grid(run.csc(v));
  const uint32_t blocks = pagerank_partial_blocks(run.csc(v));  // block sums kept

  unsigned char* p = base;
  auto take = [&](uint64_t bytes) {
    unsigned char* q = p;
    p += align256(bytes);
    return q;
  };
  double* x = reinterpret_cast<double*>(take(2 * n * 8));
  double* msg = reinterpret_cast<double*>(take(2 * n * 8));
  double* out = reinterpret_cast<double*>(take(n * 8));
  uint64_t* tomb = nullptr;
  if (tomb_in) {
    const uint64_t words = (n + 63) / 64;
    uint64_t* ids = reinterpret_cast<uint64_t*>(take(2 * words * 8));
    WC_CUDA(cudaMemcpyAsync(ids, tomb_in, words * 8, cudaMemcpyDefault, ctx.stream), ctx.detail);
    tomb = ids + words;
    WC_TRY(bits_to_locality(v, ctx.stream, ids, tomb));
  }
  const uint64_t scalar_bytes = (2 * (uint64_t)o->max_iter + 8) * 8 + 2 * (uint64_t)blocks * 8 + 64;
  double* sc = reinterpret_cast<double*>(take(scalar_bytes));
  WC_CUDA(cudaMemsetAsync(sc, 0, scalar_bytes, ctx.stream), ctx.detail);

  PrState& s = run.s;
  s = PrState{};
  s.n = (uint32_t)n;
  s.x[0] = x;
  s.x[1] = x + n;
  s.msg[0] = msg;
  s.msg[1] = msg + n;
  s.out = out;
  s.tomb = tomb;
  s.start = start;
  s.damping = o->damping;
  s.teleport = teleport;
  s.threshold = threshold;
  s.has_tol = o->has_tol != 0;
  s.delta = sc;
  s.dangling = sc + o->max_iter;
  s.partials = sc + 2 * (uint64_t)o->max_iter + 8;
  unsigned char* tail = reinterpret_cast<unsigned char*>(s.partials + 2 * blocks);
  s.counter = reinterpret_cast<unsigned*>(tail);
  s.iterations = reinterpret_cast<uint32_t*>(tail + 8);
  s.done = reinterpret_cast<int32_t*>(tail + 16);
  s.cancel = v->cancel_dev;
  s.pace = v->pace_dev;
  s.err = v->error.as<DeviceError>();
  // out = plus_first over the forward CSR: each row's out-weight, into the
  // second message buffer, then renumbered.
  PullLaunch L;
  WC_TRY(prepare_pull(ctx, v->fwd, WC_PLUS_FIRST, o->weighted, WC_F64, 1, L));
  WC_TRY(launch_pull(L, WC_F64, x, s.msg[1]));
  WC_TRY(to_locality(v, ctx.stream, s.msg[1], out));
  return cuda_status(cudaGetLastError(), ctx.detail, "pagerank setup");
}

// On an early return after work was queued on the call's stream, waits for
// that work before the locks are released, so that no kernel of this call
// still uses the shared array when the next caller takes it.
struct DrainOnExit {
  cudaStream_t stream = nullptr;
  bool armed = false;
  ~DrainOnExit() {
    if (armed) cudaStreamSynchronize(stream);
  }
};

// The solve under the device's and the version's locks.  No callback of the
// caller runs here: a progress hook that called back into this entry point
// on the same device would otherwise wait on its own lock.
static wc_status noalloc_solve(wc_version* v, const wc_call* call, const wc_pagerank_opts* o,
                               const uint64_t* tombstones, double* ranks, uint32_t* iterations,
                               wc_error_detail* detail) {
  std::lock_guard<std::mutex> device_lock(g_scratch_mu[v->device]);
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), detail);
  if (!g_scratch_addr[v->device]) {
    void* addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_pagerank_scratch);
    if (e != cudaSuccess) return cuda_status(e, detail, "cudaGetSymbolAddress");
    if (!addr) {
      set_message(detail, "cudaGetSymbolAddress gave no address for the fixed scratch");
      return WC_CUDA_ERROR;
    }
    g_scratch_addr[v->device] = addr;
  }
  // No events, and no progress hook inside the locks.
  wc_call plain{};
  if (call) {
    plain = *call;
    plain.flags &= ~WC_CALL_TIMING;
    plain.progress = nullptr;
  }
  Ctx ctx(v, call ? &plain : nullptr);
  if (ctx.cancelled()) return WC_CANCELLED;
  DrainOnExit drain;  // declared after the locks: runs before they are released
  drain.stream = ctx.stream;
  drain.armed = true;
  WC_TRY(ctx.begin());
  PageRankRun run;
  WC_TRY(static_setup(ctx, run, o, tombstones,
                      static_cast<unsigned char*>(g_scratch_addr[v->device])));
  WC_TRY(run.run(ctx));
  WC_TRY(ctx.finish());
  double margin = 0.0;
  WC_TRY(run.result(ctx, ranks, iterations, &margin));
  drain.armed = false;
  v->last_margin = margin;
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_pagerank_noalloc(wc_version* v, const wc_call* call, const wc_pagerank_opts* o,
                              const uint64_t* tombstones, double* ranks, uint32_t* iterations) {
  if (!v || !o || !ranks) return WC_INVALID_ARGUMENT;
  wc_error_detail* detail = call ? call->detail : nullptr;
  if (v->device < 0 || v->device >= kMaxDevices) {
    set_message(detail, "device %d is beyond the %d devices served", v->device, kMaxDevices);
    return WC_UNSUPPORTED;
  }
  if (o->seed) {
    set_message(detail, "a personalised PageRank needs per-call memory; use wc_pagerank");
    return WC_UNSUPPORTED;
  }
  const uint32_t blocks = pagerank_partial_blocks(v->loc.csc);
  const uint64_t need = static_bytes(v->n, o->max_iter, blocks, tombstones != nullptr);
  if (need > kStaticScratchBytes) {
    if (detail) {
      detail->requested = need;
      detail->limit = kStaticScratchBytes;
    }
    set_message(detail, "%llu nodes and %u iterations need %llu bytes of fixed scratch; the limit is %llu",
                (unsigned long long)v->n, o->max_iter, (unsigned long long)need,
                (unsigned long long)kStaticScratchBytes);
    return WC_WORKING_SET;
  }
  // The progress hook runs outside the locks, before and after the solve.
  const bool hook = call && call->progress;
  if (hook) call->progress(call->progress_context, "iterating", 0, o->max_iter);
  const wc_status st = noalloc_solve(v, call, o, tombstones, ranks, iterations, detail);
  if (st == WC_OK && hook)
    call->progress(call->progress_context, "iterating", iterations ? *iterations : 0, o->max_iter);
  return st;
}

}  // extern "C"
