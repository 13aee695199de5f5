// runtime.cuh — the backend's host runtime: device memory charged to a
// budget before it is allocated, the version handle holding the device CSR
// and CSC, and the per-call context (stream, error word, cancellation).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <thread>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/warren_cuda.h"

namespace wc {

// Every kernel launch of the library is counted (wc_kernel_launches), so a
// caller can see that its work ran here and how many launches it took.
extern std::atomic<uint64_t> g_launches;
inline void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ------------------------------------------------------------------ budget
// compute/memory.rs:31-227: every buffer is charged before it is allocated;
// a charge past the limit is refused with what was asked and what is held.
}  // namespace wc

struct wc_budget {
  uint64_t limit;
  std::atomic<uint64_t> in_use{0};
  std::atomic<uint64_t> peak{0};
  std::mutex mu;
  // The creator's reference and one per version charged to it: a version
  // keeps its budget alive until its own buffers are freed, whatever order
  // the caller releases them in.
  std::atomic<int> refs{1};
};

namespace wc {

inline void budget_retain(wc_budget* b) {
  if (b) b->refs.fetch_add(1);
}
inline void budget_release(wc_budget* b) {
  if (b && b->refs.fetch_sub(1) == 1) delete b;
}

// A version's reference to its budget, released after every other member
// of the version (it is declared first), so its buffers uncharge a live one.
struct BudgetRef {
  wc_budget* b = nullptr;
  BudgetRef() = default;
  BudgetRef(const BudgetRef&) = delete;
  BudgetRef& operator=(const BudgetRef&) = delete;
  void hold(wc_budget* x) {
    budget_retain(x);
    budget_release(b);
    b = x;
  }
  ~BudgetRef() { budget_release(b); }
};

inline void set_message(wc_error_detail* d, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
inline void set_message(wc_error_detail* d, const char* fmt, ...) {
  if (!d) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(d->message, sizeof d->message, fmt, ap);
  va_end(ap);
}

// A failed CUDA call: WC_CUDA_ERROR with the error code in the detail.
inline wc_status cuda_status(cudaError_t e, wc_error_detail* d, const char* where) {
  if (e == cudaSuccess) return WC_OK;
  if (d) {
    d->cuda_error = (int32_t)e;
    set_message(d, "%s: %s", where, cudaGetErrorString(e));
  }
  if (e == cudaErrorMemoryAllocation) return WC_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return WC_NO_DEVICE;
  return WC_CUDA_ERROR;
}

#define WC_TRY(expr)                 \
  do {                               \
    wc_status _s = (expr);           \
    if (_s != WC_OK) return _s;      \
  } while (0)

#define WC_CUDA(expr, detail)                                       \
  do {                                                              \
    cudaError_t _e = (expr);                                        \
    if (_e != cudaSuccess) return ::wc::cuda_status(_e, detail, #expr); \
  } while (0)

inline wc_status charge(wc_budget* b, uint64_t bytes, wc_error_detail* d) {
  if (!b) return WC_OK;
  std::lock_guard<std::mutex> lock(b->mu);
  uint64_t used = b->in_use.load();
  if (bytes > b->limit || used > b->limit - bytes) {
    if (d) {
      d->requested = bytes;
      d->in_use = used;
      d->limit = b->limit;
      set_message(d, "compute memory limit exceeded: %llu bytes requested, %llu of %llu in use",
                  (unsigned long long)bytes, (unsigned long long)used,
                  (unsigned long long)b->limit);
    }
    return WC_MEMORY_LIMIT;
  }
  b->in_use.store(used + bytes);
  if (used + bytes > b->peak.load()) b->peak.store(used + bytes);
  return WC_OK;
}

inline void uncharge(wc_budget* b, uint64_t bytes) {
  if (!b) return;
  std::lock_guard<std::mutex> lock(b->mu);
  b->in_use.store(b->in_use.load() - bytes);
}

// A device buffer charged to a budget for its lifetime.
struct DevBuf {
  void* ptr = nullptr;
  uint64_t bytes = 0;
  wc_budget* budget = nullptr;

  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      budget = o.budget;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }

  void release() {
    if (ptr) {
      cudaFree(ptr);
      uncharge(budget, bytes);
    }
    ptr = nullptr;
    bytes = 0;
  }

  wc_status alloc(wc_budget* b, uint64_t n, wc_error_detail* d) {
    release();
    if (n == 0) n = 16;
    n = (n + 255) & ~uint64_t(255);
    WC_TRY(charge(b, n, d));
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
      uncharge(b, n);
      ptr = nullptr;
      cudaGetLastError();
      if (d) {
        d->requested = n;
        set_message(d, "out of memory allocating %llu bytes", (unsigned long long)n);
      }
      return WC_OUT_OF_MEMORY;
    }
    bytes = n;
    budget = b;
    return WC_OK;
  }

  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Where a device buffer of an operand comes from: the caller's own device
// pointer, or a staging copy of a host operand.
inline bool is_device_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The device error word a kernel raises: the first status wins (atomicCAS
// from 0); `aux` carries a node id or a count where the status has one.
struct DeviceError {
  int32_t status;
  int32_t pad;
  uint64_t aux;
};

// The version's pinned staging area: the device error word's read-back,
// then a small plan area, then a payload area.
constexpr uint64_t kStageBytes = 65536;
constexpr uint64_t kStageError = 0;
constexpr uint64_t kStagePlan = 64;
constexpr uint64_t kStagePlanBytes = 4032;
constexpr uint64_t kStagePayload = kStagePlan + kStagePlanBytes;

// ------------------------------------------------------------------ schedule
// The row-split schedule of one CSR orientation for the pull kernels: rows
// grouped into warp tiles (at most kTileRows consecutive rows, at most
// kTileEntries entries, none longer than that), and each longer row split
// into pieces of at most kPieceEntries entries whose partial results are
// combined in piece order by the last piece to finish.  Every unit is at
// most 256 entries, so warps taking units round-robin stay balanced.
constexpr uint32_t kTileRows = 32;
constexpr uint32_t kTileEntries = 256;
constexpr uint32_t kPieceEntries = 256;
// Tail padding of the device CSR arrays (bulk copies read up to 16-byte
// boundaries).
constexpr uint64_t kBulkPad = 16;

struct Unit {
  // tile: rows [a, b) holding c (<= 256) entries from entry d;
  // piece: row a, entries [b, d), c = 1<<31 | slot.
  uint32_t a, b, c, d;
};

struct Schedule {
  DevBuf units;       // Unit[count]
  DevBuf counters;    // u32[slots]: arrivals per long row (indexed by its first slot)
  DevBuf carry;       // the pieces' partial results, kCarryBytesPerSlot per slot
  DevBuf long_list;   // uint4[long_rows]: each long row, its first slot and piece count
  DevBuf row_masks;   // u32[count]: a tile's rows that hold entries (bit r: row a + r)
  uint32_t count = 0;
  uint32_t slots = 0;
  uint32_t long_rows = 0;
  uint32_t tiles = 0;
};

// One CSR orientation on the device: u32 offsets and targets, f64 weights
// (absent when unweighted) and, when every weight is an integer in int32
// range, an int32 copy for the integer semirings.
struct DevCsr {
  DevBuf offsets, targets, weights, iweights;
  Schedule schedule;
  uint32_t max_degree = 0;
};

// The reverse CSR in locality order (locality.cu): nodes renumbered by
// out-degree, largest first; perm maps a dense id to its new number and
// order a new number back to the dense id.
struct Locality {
  DevBuf perm, order;  // u32[n] each
  DevCsr csc;
};

}  // namespace wc

// The handle: one version's device copy, keyed by (graph, version).
struct wc_version {
  wc::BudgetRef budget_ref;  // first: released last
  uint64_t graph_id = 0, version = 0;
  uint64_t n = 0, m = 0;
  int device = 0;
  bool weighted = false;
  bool integral = false;
  int64_t max_abs_iweight = -1;  // max |w| when every weight is an i32 (1 unweighted), else -1
  bool symmetric = false;
  wc_budget* budget = nullptr;
  cudaStream_t stream = nullptr;
  wc::DevCsr fwd, rev;
  wc::Locality loc;                    // rev renumbered for the pull solvers
  bool reverse_given = false;          // the caller uploaded a reverse CSR
  std::vector<uint64_t> host_offsets;  // forward offsets, for truncated-BFS stats
  std::vector<uint64_t> host_rev_offsets;
  wc::DevBuf error;                    // DeviceError
  int32_t* cancel_host = nullptr;      // pinned, mapped: the device reads it
  int32_t* cancel_dev = nullptr;
  volatile uint32_t* pace_host = nullptr;  // mapped: [0] iterations done, [1] stopped
  uint32_t* pace_dev = nullptr;
  // Pinned host staging (wc::kStage*): small per-call uploads and
  // read-backs, which captured graphs may also copy from and to.
  uint8_t* stage_host = nullptr;
  uint8_t* stage_dev = nullptr;  // the same memory, mapped for kernels
  std::recursive_mutex mu;             // calls on one handle run one at a time
  double last_margin = 0.0;
  std::map<uint64_t, wc_schedule> tuned;  // (kind << 32 | width) -> schedule
  // Scratch kept between calls (charged to the budget while held), so a
  // call allocates only when it needs more than the last one did.  Calls on
  // one handle are serialised; asynchronous ones must share one stream.
  std::map<int, wc::DevBuf> pool;
  // Kernel-group timings of the last call made with WC_CALL_TIMING.
  std::map<std::string, std::pair<double, uint32_t>> timings;
  // Executable CUDA graphs of fixed launch sequences, by shape (see
  // Ctx::run_captured); destroyed with the version.
  std::map<std::string, cudaGraphExec_t> graphs;
  // The launch arguments each of those graphs was captured with (run_cached).
  std::map<std::string, std::string> graph_args;
  // Cursors open over the version (wc_bfs_cursor): it is not released
  // while any is.
  std::atomic<uint32_t> cursors{0};
};

namespace wc {

// The pool's tags: one buffer per role.
enum PoolTag {
  POOL_X = 1, POOL_Y, POOL_MASK, POOL_XCOPY, POOL_SEED,
  POOL_PR_X, POOL_PR_MSG, POOL_PR_OUT, POOL_PR_SHARES, POOL_PR_TOMB, POOL_PR_SCALARS,
  POOL_BFS_DEPTH, POOL_BFS_VIA, POOL_BFS_Q0, POOL_BFS_Q1, POOL_BFS_FBITS, POOL_BFS_COUNTERS,
  POOL_BFS_FILTER, POOL_BFS_FLAGS, POOL_BFS_BIG = 30, POOL_BFS_ROWS, POOL_BFS_SCAN,
  POOL_BATCH_0 = 40, POOL_BATCH_1, POOL_BATCH_2, POOL_BATCH_3, POOL_BATCH_4, POOL_BATCH_5,
  POOL_BATCH_6, POOL_BATCH_7, POOL_BATCH_8, POOL_BATCH_9, POOL_BATCH_10, POOL_BATCH_11,
  POOL_EIG_0 = 60, POOL_EIG_1, POOL_EIG_2, POOL_EIG_3, POOL_EIG_4, POOL_EIG_5, POOL_EIG_6,
  POOL_EIG_7, POOL_EIG_8, POOL_EIG_9,
  POOL_ADJ_0 = 80, POOL_ADJ_1, POOL_ADJ_2, POOL_ADJ_3, POOL_ADJ_4, POOL_ADJ_5, POOL_ADJ_6,
  POOL_ADJ_7, POOL_ADJ_8, POOL_ADJ_9,
  POOL_TOPK_0 = 100, POOL_TOPK_1,
  // Buffers the batched BFS keeps all-zero between calls; no other role
  // may share them.
  POOL_MSBFS_NACC = 110, POOL_MSBFS_ACC, POOL_MSBFS_TOUCHED, POOL_MSBFS_PULLED,
  // The 32-bit batched min-plus's long-row minima, kept at i32::MAX.
  POOL_MINPLUS32_NACC = 120,
  POOL_WCC_PARENT = 130, POOL_WCC_FLAG, POOL_WCC_LABELS,
  POOL_SPMM_CARRY = 140,
  POOL_CENT_TOTALS = 150, POOL_CENT_FLAG, POOL_CENT_SOURCES, POOL_CENT_CAPS, POOL_CENT_LIST,
  POOL_CENT_TOMB, POOL_CENT_VALUES,
  POOL_VEC_PARTIAL = 160, POOL_VEC_RESULT,
  POOL_MAP_PROGRAM = 170, POOL_MAP_ERROR, POOL_MAP_OUT,
  POOL_MAP_OPERAND_0 = 180,  // .. 195: one per operand
  POOL_BC_SIGMA = 200, POOL_BC_DELTA, POOL_BC_TOTAL, POOL_BC_REACHED, POOL_BC_FLAG,
  POOL_BC_SOURCES, POOL_BC_CAPS, POOL_BC_LIST, POOL_BC_TOMB, POOL_BC_VALUES, POOL_BC_CARRY,
  // A row-partitioned search's part: held from its begin to its end.
  POOL_PART_VISITED = 220, POOL_PART_DEPTH, POOL_PART_SUMS, POOL_PART_STARTS,
};

// A call's context: the stream, the caller's detail and cancellation.
struct Ctx {
  wc_version* v;
  const wc_call* call;
  cudaStream_t stream;
  wc_budget* budget;                  // the version's: the pool's device memory
  wc_budget* call_budget = nullptr;   // the call's own (wc_call.memory), if any
  uint64_t call_charged = 0;          // bytes charged to it by this call
  wc_error_detail* detail;
  bool async;
  uint32_t timeout_ms;

  bool timing = false;
  bool capturing = false;  // the stream is being captured by run_captured
  bool device_error = false;  // finish() returned a status a kernel raised
  struct Timer {
    std::string name;
    cudaEvent_t a, b;
    uint64_t launches;
  };
  std::vector<Timer> timers;
  std::vector<size_t> open;  // timers begun and not yet ended (phases nest)

  Ctx(wc_version* ver, const wc_call* c)
      : v(ver), call(c), stream(ver->stream), budget(ver->budget), detail(nullptr),
        async(false), timeout_ms(600000) {
    if (c) {
      if (c->stream) stream = (cudaStream_t)c->stream;
      if (c->memory && c->memory != ver->budget) call_budget = c->memory;
      detail = c->detail;
      async = (c->flags & WC_CALL_ASYNC) != 0;
      timing = (c->flags & WC_CALL_TIMING) != 0;
      if (c->timeout_ms) timeout_ms = c->timeout_ms;
    }
  }
  ~Ctx() {
    if (call_budget && call_charged) uncharge(call_budget, call_charged);
    for (Timer& t : timers) {
      cudaEventDestroy(t.a);
      cudaEventDestroy(t.b);
    }
  }

  // Brackets a kernel group with events when the caller asked for timing.
  void phase_begin(const char* name) {
    if (!timing) return;
    Timer t{name, nullptr, nullptr, g_launches.load()};
    cudaEventCreate(&t.a);
    cudaEventCreate(&t.b);
    record(t.a);
    open.push_back(timers.size());
    timers.push_back(t);
  }
  void phase_end() {
    if (!timing || open.empty()) return;
    Timer& t = timers[open.back()];
    open.pop_back();
    record(t.b);
    t.launches = g_launches.load() - t.launches;
  }
  // Inside a capture the record becomes a graph node that still times.
  void record(cudaEvent_t e) {
    if (capturing) cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal);
    else cudaEventRecord(e, stream);
  }

  // Queues `enqueue`'s launch sequence (which must allocate nothing and
  // wait for nothing) as a CUDA graph: the sequence is captured from the
  // stream, the version's executable graph for `key` is updated in place to
  // it (instantiated the first time, or when the update is refused), and
  // that graph is launched.  A stream the caller is already capturing gets
  // the sequence directly, as part of the caller's graph.
  template <class F> wc_status run_captured(const std::string& key, F&& enqueue) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (!stream || cudaStreamIsCapturing(stream, &cs) != cudaSuccess ||
        cs != cudaStreamCaptureStatusNone)
      return enqueue();
    cudaGraphExec_t exec = nullptr;
    v->graph_args.erase(key);
    WC_TRY(capture(key, enqueue, &exec));
    return cuda_status(cudaGraphLaunch(exec, stream), detail, "cudaGraphLaunch");
  }

  // run_captured for a sequence whose launches are fully described by
  // `args` (every kernel argument, copy and size, flattened): when the
  // version's graph for `key` was captured with the same `args` it is
  // launched as it stands, with no capture.  What changes from call to call
  // must then come through memory (a pinned staging copy in the graph).
  template <class F> wc_status run_cached(const std::string& key, const std::string& args,
                                          F&& enqueue) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (!stream || cudaStreamIsCapturing(stream, &cs) != cudaSuccess ||
        cs != cudaStreamCaptureStatusNone)
      return enqueue();
    auto it = v->graphs.find(key);
    auto at = v->graph_args.find(key);
    if (it != v->graphs.end() && it->second && at != v->graph_args.end() && at->second == args)
      return cuda_status(cudaGraphLaunch(it->second, stream), detail, "cudaGraphLaunch");
    v->graph_args.erase(key);
    cudaGraphExec_t exec = nullptr;
    WC_TRY(capture(key, enqueue, &exec));
    v->graph_args[key] = args;
    return cuda_status(cudaGraphLaunch(exec, stream), detail, "cudaGraphLaunch");
  }

  // Captures `enqueue`'s launch sequence from the stream (which no one may
  // be capturing already) into the version's executable graph for `key`,
  // updated in place or instantiated, and returns it without launching it.
  template <class F> wc_status capture(const std::string& key, F&& enqueue, cudaGraphExec_t* out) {
    WC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), detail);
    capturing = true;
    const wc_status st = enqueue();
    capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t ended = cudaStreamEndCapture(stream, &graph);
    if (st != WC_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (ended != cudaSuccess) return cuda_status(ended, detail, "cudaStreamEndCapture");
    cudaGraphExec_t& exec = v->graphs[key];
    if (exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(exec, graph, &info) != cudaSuccess) {
        (void)cudaGetLastError();
        cudaGraphExecDestroy(exec);
        exec = nullptr;
      }
    }
    if (!exec) {
      const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
      if (e != cudaSuccess) {
        exec = nullptr;
        cudaGraphDestroy(graph);
        return cuda_status(e, detail, "cudaGraphInstantiate");
      }
    }
    cudaGraphDestroy(graph);
    *out = exec;
    return WC_OK;
  }

  void collect_timings() {
    if (!timing) return;
    v->timings.clear();
    for (Timer& t : timers) {
      float ms = 0.0f;
      if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
        auto& slot = v->timings[t.name];
        slot.first += ms;
        slot.second += (uint32_t)t.launches;
      }
    }
  }

  bool cancelled() const { return call && call->cancel && *call->cancel; }

  // Pooled scratch of at least `bytes` under `tag` (contents undefined).
  // The device allocation belongs to the version's pool and is charged to
  // the version's budget while the pool holds it.  A call given its own
  // budget (wc_call.memory) is also charged the bytes it uses, for the
  // call's duration, as the reference charges a call's ComputeMemory; a
  // refusal there is WC_MEMORY_LIMIT before anything is allocated.
  wc_status scratch(int tag, uint64_t bytes, DevBuf** out) {
    if (call_budget) {
      WC_TRY(charge(call_budget, bytes, detail));
      call_charged += bytes;
    }
    DevBuf& b = v->pool[tag];
    if (b.bytes < bytes) {
      b.release();
      WC_TRY(b.alloc(budget, bytes + bytes / 8, detail));
    }
    *out = &b;
    return WC_OK;
  }

  void progress(const char* phase, uint64_t done, uint64_t total) const {
    if (call && call->progress) call->progress(call->progress_context, phase, done, total);
  }

  // Clears the device error word and the device-visible cancel flag.
  wc_status begin() {
    *v->cancel_host = 0;
    WC_CUDA(cudaMemsetAsync(v->error.ptr, 0, sizeof(DeviceError), stream), detail);
    return WC_OK;
  }

  // Waits for the stream, polling the caller's cancel word every 50 µs and
  // passing it on to the device (kernels that loop read it and stop).  Then
  // reads the device error word.
  wc_status finish() {
    // The device error word comes back behind the call's work, so one wait
    // covers both.
    WC_CUDA(cudaMemcpyAsync(v->stage_host + kStageError, v->error.ptr, sizeof(DeviceError),
                            cudaMemcpyDeviceToHost, stream), detail);
    auto start = std::chrono::steady_clock::now();
    bool cancel = false, timed_out = false;
    for (;;) {
      cudaError_t q = cudaStreamQuery(stream);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return cuda_status(q, detail, "cudaStreamQuery");
      if (!cancel && cancelled()) {
        cancel = true;
        *v->cancel_host = 1;
      }
      auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                    std::chrono::steady_clock::now() - start).count();
      if (!timed_out && (uint64_t)ms > timeout_ms) {
        timed_out = true;
        *v->cancel_host = 1;
      }
      if (ms >= 2) std::this_thread::sleep_for(std::chrono::microseconds(20));
      else std::this_thread::yield();
    }
    // A cancel raised while the call ran is reported even when the device
    // finished first (the reference's last check before it returns).
    if (!cancel && cancelled()) cancel = true;
    collect_timings();
    DeviceError e;
    std::memcpy(&e, v->stage_host + kStageError, sizeof e);
    if (cancel) return WC_CANCELLED;
    if (timed_out) return WC_DEVICE_TIMEOUT;
    if (e.status != 0) {
      if (detail) detail->node = e.aux;
      device_error = true;
      return (wc_status)e.status;
    }
    return WC_OK;
  }

};

}  // namespace wc
