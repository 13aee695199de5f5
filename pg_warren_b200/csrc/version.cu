// version.cu — budgets, the version handle and its upload: the device copy
// of a built version's CSR and reverse CSR (graph/csr/mod.rs:38-237,
// graph_csr.rs:15-55), with the row-split schedules the pull kernels walk.
#include <algorithm>
#include <cstdlib>
#include <memory>
#include <thread>

#include "pagerank.h"
#include "product.h"
#include "runtime.cuh"
#include "upload.h"

namespace wc {

std::atomic<uint64_t> g_launches{0};

// The reverse CSR by a counting transpose: in-degrees, then a scatter while
// sources are scanned in order, so each reverse row comes out ascending
// (graph/csr/transpose.rs:14-44).
void host_transpose(uint64_t n, uint64_t m, const uint64_t* off, const uint32_t* tgt,
                    const double* w, uint64_t* roff, uint32_t* rtgt, double* rw) {
  std::fill(roff, roff + n + 1, 0);
  for (uint64_t e = 0; e < m; e++) roff[tgt[e] + 1]++;
  for (uint64_t i = 0; i < n; i++) roff[i + 1] += roff[i];
  std::vector<uint64_t> cursor(roff, roff + n);
  for (uint64_t s = 0; s < n; s++)
    for (uint64_t e = off[s]; e < off[s + 1]; e++) {
      uint64_t p = cursor[tgt[e]]++;
      rtgt[p] = (uint32_t)s;
      if (w && rw) rw[p] = w[e];
    }
}

// The schedule of one orientation: tiles of up to kTileRows consecutive
// rows with at most kTileEntries entries, and the longer rows' pieces.
static void build_units(uint64_t n, const uint64_t* off, std::vector<Unit>& units,
                        uint32_t& slots, uint32_t& long_rows, uint32_t& tiles, uint32_t& max_deg) {
  units.clear();
  slots = long_rows = tiles = max_deg = 0;
  uint64_t r = 0;
  while (r < n) {
    uint64_t deg = off[r + 1] - off[r];
    max_deg = std::max<uint32_t>(max_deg, (uint32_t)deg);
    if (deg > kTileEntries) {
      long_rows++;
      for (uint64_t e = off[r]; e < off[r + 1]; e += kPieceEntries) {
        uint64_t end = std::min<uint64_t>(off[r + 1], e + kPieceEntries);
        units.push_back(Unit{(uint32_t)r, (uint32_t)e, (1u << 31) | slots, (uint32_t)end});
        slots++;
      }
      r++;
      continue;
    }
    uint64_t start = r, entries = 0;
    while (r < n && r - start < kTileRows) {
      uint64_t d = off[r + 1] - off[r];
      if (d > kTileEntries || entries + d > kTileEntries) break;
      max_deg = std::max<uint32_t>(max_deg, (uint32_t)d);
      entries += d;
      r++;
    }
    units.push_back(Unit{(uint32_t)start, (uint32_t)r, (uint32_t)entries, (uint32_t)off[start]});
    tiles++;
  }
}

// One orientation's arrays, copied from the host (u32 offsets).
static wc_status put_csr(wc_version* v, DevCsr& d, const uint64_t* off, const uint32_t* tgt,
                         const double* w, wc_error_detail* detail) {
  const uint64_t n = v->n, m = v->m;
  std::vector<uint32_t> off32(n + 1);
  for (uint64_t i = 0; i <= n; i++) off32[i] = (uint32_t)off[i];
  // 16 bytes of tail padding on each array: the pull's bulk copies widen
  // their spans to 16-byte boundaries.
  WC_TRY(d.offsets.alloc(v->budget, (n + 1) * 4 + kBulkPad, detail));
  WC_TRY(d.targets.alloc(v->budget, m * 4 + kBulkPad, detail));
  WC_CUDA(cudaMemcpyAsync(d.offsets.ptr, off32.data(), (n + 1) * 4, cudaMemcpyHostToDevice,
                          v->stream), detail);
  if (m)
    WC_CUDA(cudaMemcpyAsync(d.targets.ptr, tgt, m * 4, cudaMemcpyHostToDevice, v->stream), detail);
  if (w) {
    WC_TRY(d.weights.alloc(v->budget, m * 8 + kBulkPad, detail));
    if (m)
      WC_CUDA(cudaMemcpyAsync(d.weights.ptr, w, m * 8, cudaMemcpyHostToDevice, v->stream), detail);
  }
  // The copies read the host staging of the offsets: wait for them.
  return cuda_status(cudaStreamSynchronize(v->stream), detail, "version upload");
}

// The schedule of one orientation from its host offsets.
wc_status put_schedule(wc_version* v, DevCsr& d, const std::vector<uint64_t>& off,
                              wc_error_detail* detail) {
  std::vector<Unit> units;
  Schedule& s = d.schedule;
  build_units(v->n, off.data(), units, s.slots, s.long_rows, s.tiles, d.max_degree);
  s.count = (uint32_t)units.size();
  WC_TRY(s.units.alloc(v->budget, std::max<size_t>(units.size(), 1) * sizeof(Unit), detail));
  if (!units.empty())
    WC_CUDA(cudaMemcpy(s.units.ptr, units.data(), units.size() * sizeof(Unit),
                       cudaMemcpyHostToDevice), detail);
  WC_TRY(s.counters.alloc(v->budget, (uint64_t)std::max<uint32_t>(s.slots, 1) * 4, detail));
  WC_CUDA(cudaMemset(s.counters.ptr, 0, (uint64_t)std::max<uint32_t>(s.slots, 1) * 4), detail);
  WC_TRY(s.carry.alloc(v->budget, (uint64_t)std::max<uint32_t>(s.slots, 1) * kCarryBytesPerSlot,
                       detail));
  // The long rows, for kernels that combine their pieces in a pass of their
  // own: (row, first slot, pieces) in row order.
  std::vector<uint32_t> longs;
  longs.reserve(4 * (size_t)s.long_rows);
  for (size_t u = 0; u < units.size(); u++) {
    const Unit& d = units[u];
    if ((d.c >> 31) == 0) continue;
    if (u > 0 && (units[u - 1].c >> 31) != 0 && units[u - 1].a == d.a) continue;
    const uint64_t deg = off[d.a + 1] - off[d.a];
    longs.insert(longs.end(), {d.a, d.c & 0x7fffffffu, (uint32_t)((deg + kPieceEntries - 1) / kPieceEntries), 0u});
  }
  WC_TRY(s.long_list.alloc(v->budget, std::max<size_t>(longs.size(), 4) * 4, detail));
  if (!longs.empty())
    WC_CUDA(cudaMemcpy(s.long_list.ptr, longs.data(), longs.size() * 4, cudaMemcpyHostToDevice),
            detail);
  // Per tile, its rows that hold entries (a piece's row always does).
  std::vector<uint32_t> masks(units.size(), 1u);
  for (size_t u = 0; u < units.size(); u++) {
    const Unit& d = units[u];
    if ((d.c >> 31) != 0) continue;
    uint32_t m = 0;
    for (uint32_t r = d.a; r < d.b; r++)
      if (off[r + 1] > off[r]) m |= 1u << (r - d.a);
    masks[u] = m;
  }
  WC_TRY(s.row_masks.alloc(v->budget, std::max<size_t>(masks.size(), 1) * 4, detail));
  if (!masks.empty())
    WC_CUDA(cudaMemcpy(s.row_masks.ptr, masks.data(), masks.size() * 4, cudaMemcpyHostToDevice),
            detail);
  return WC_OK;
}

wc_status wc_device_check(wc_error_detail* detail) {
  int device = 0, count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_message(detail, "no CUDA device");
    return WC_NO_DEVICE;
  }
  WC_CUDA(cudaGetDevice(&device), detail);
  cudaDeviceProp prop;
  WC_CUDA(cudaGetDeviceProperties(&prop, device), detail);
  if (prop.major < 10) {
    set_message(detail, "device %d is sm_%d%d; this library is built for sm_100a", device,
                prop.major, prop.minor);
    return WC_NO_DEVICE;
  }
  return WC_OK;
}

wc_status finish_version(wc_version* v, wc_error_detail* detail) {
  WC_TRY(device_weight_facts(v, detail));
  WC_TRY(device_symmetric(v, detail));
  WC_TRY(put_schedule(v, v->fwd, v->host_offsets, detail));
  WC_TRY(put_schedule(v, v->rev, v->host_rev_offsets, detail));
  WC_TRY(device_locality(v, detail));
  WC_TRY(v->error.alloc(v->budget, sizeof(DeviceError), detail));
  WC_CUDA(cudaMemset(v->error.ptr, 0, sizeof(DeviceError)), detail);
  // Four mapped words: the cancel word, then the pacing words (iterations
  // completed, done) that iterative kernels report to the host.
  WC_CUDA(cudaHostAlloc((void**)&v->cancel_host, 4 * sizeof(int32_t), cudaHostAllocMapped), detail);
  for (int q = 0; q < 4; q++) v->cancel_host[q] = 0;
  WC_CUDA(cudaHostGetDevicePointer((void**)&v->cancel_dev, v->cancel_host, 0), detail);
  v->pace_host = reinterpret_cast<volatile uint32_t*>(v->cancel_host + 1);
  v->pace_dev = reinterpret_cast<uint32_t*>(v->cancel_dev + 1);
  WC_CUDA(cudaHostAlloc((void**)&v->stage_host, kStageBytes, cudaHostAllocMapped), detail);
  WC_CUDA(cudaHostGetDevicePointer((void**)&v->stage_dev, v->stage_host, 0), detail);
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

const char* wc_status_name(wc_status s) {
  switch (s) {
    case WC_OK: return "ok";
    case WC_MEMORY_LIMIT: return "compute memory limit exceeded";
    case WC_OUT_OF_MEMORY: return "out of memory";
    case WC_DTYPE_MISMATCH: return "element type mismatch";
    case WC_ID_SPACE_MISMATCH: return "vector id space does not match the graph";
    case WC_WIDTH_MISMATCH: return "vector width mismatch";
    case WC_UNKNOWN_SEMIRING: return "unknown semiring";
    case WC_UNKNOWN_BINARY_OP: return "unknown binary operator";
    case WC_ZERO_WIDTH: return "a vector's width must be at least 1";
    case WC_CANCELLED: return "compute cancelled";
    case WC_BIGINT_OUT_OF_RANGE: return "bigint out of range";
    case WC_FLOAT_OVERFLOW: return "value out of range: overflow";
    case WC_FLOAT_UNDERFLOW: return "value out of range: underflow";
    case WC_DIVISION_BY_ZERO: return "division by zero";
    case WC_NODE_OUTSIDE_ID_SPACE: return "node outside the id space";
    case WC_NODE_FILTER_ID_SPACE: return "node filter over another id space";
    case WC_REVERSE_CSR_MISSING: return "the reverse CSR is missing";
    case WC_NOT_SYMMETRIC: return "the matrix is not symmetric";
    case WC_SEGMENT_TRUNCATED: return "segment truncated";
    case WC_SEGMENT_MAGIC: return "not a pg_warren segment";
    case WC_SEGMENT_FORMAT: return "unsupported segment format";
    case WC_SEGMENT_KIND: return "segment kind mismatch";
    case WC_SEGMENT_RESERVED: return "segment reserved byte is not 0";
    case WC_SEGMENT_WIDTH: return "segment element width mismatch";
    case WC_SEGMENT_LENGTH: return "segment payload length mismatch";
    case WC_OFFSETS_LENGTH: return "CSR offsets length mismatch";
    case WC_FIRST_OFFSET_NOT_ZERO: return "CSR offsets do not start at 0";
    case WC_STORED_ROWS_NOT_ASCENDING: return "CSR stored rows not ascending";
    case WC_STORED_ROW_OUTSIDE_ID_SPACE: return "CSR stores a row outside the id space";
    case WC_STORED_ROW_EMPTY: return "CSR stores a row without targets";
    case WC_OFFSETS_NOT_MONOTONE: return "CSR offsets decrease";
    case WC_FINAL_OFFSET: return "CSR final offset mismatch";
    case WC_TARGET_OUTSIDE_ID_SPACE: return "CSR target outside the id space";
    case WC_ROW_NOT_SORTED: return "CSR row not strictly ascending";
    case WC_WEIGHTS_LENGTH: return "CSR weights length mismatch";
    case WC_NON_POSITIVE_DEGREE: return "a node with an edge has a non-positive degree";
    case WC_EIGENPAIR_COUNT: return "eigenpair count out of range";
    case WC_WORKING_SET: return "the eigenproblem's working set does not fit the compute memory";
    case WC_NOT_FINITE: return "a value overflowed";
    case WC_INVALID_ARGUMENT: return "invalid argument";
    case WC_UNSUPPORTED: return "not served by this backend";
    case WC_CUDA_ERROR: return "CUDA error";
    case WC_DEVICE_TIMEOUT: return "a device wait timed out";
    case WC_NO_DEVICE: return "no usable device";
  }
  return "unknown status";
}

wc_status wc_budget_create(uint64_t limit, wc_budget** out) {
  if (!out) return WC_INVALID_ARGUMENT;
  auto* b = new wc_budget;
  b->limit = limit;
  *out = b;
  return WC_OK;
}

void wc_budget_destroy(wc_budget* b) { budget_release(b); }
uint64_t wc_budget_in_use(const wc_budget* b) { return b ? b->in_use.load() : 0; }
uint64_t wc_budget_peak(const wc_budget* b) { return b ? b->peak.load() : 0; }

wc_status wc_version_upload(uint64_t graph_id, uint64_t version, const wc_csr_host* csr,
                            wc_budget* budget, const wc_call* call, wc_version** out) {
  wc_error_detail* detail = call ? call->detail : nullptr;
  if (!csr || !out || !csr->offsets || (csr->edges && !csr->targets)) return WC_INVALID_ARGUMENT;
  *out = nullptr;
  if (csr->id_space >= (1ull << 32) || csr->edges >= (1ull << 32)) {
    set_message(detail, "id spaces and edge counts of 2^32 or more are not served");
    return WC_UNSUPPORTED;
  }
  WC_TRY(wc_device_check(detail));
  const uint64_t n = csr->id_space, m = csr->edges;
  if (csr->offsets[0] != 0 || csr->offsets[n] != m) return WC_INVALID_ARGUMENT;
  for (uint64_t e = 0; e < m; e++)
    if (csr->targets[e] >= n) {
      if (detail) detail->node = csr->targets[e];
      return WC_NODE_OUTSIDE_ID_SPACE;
    }
  if (csr->reverse_offsets && (!csr->reverse_targets || (csr->weights && !csr->reverse_weights)))
    return WC_INVALID_ARGUMENT;
  std::unique_ptr<wc_version> v(new wc_version);
  v->graph_id = graph_id;
  v->version = version;
  v->n = n;
  v->m = m;
  v->budget = budget;
  v->budget_ref.hold(budget);
  v->weighted = csr->weights != nullptr;
  WC_CUDA(cudaGetDevice(&v->device), detail);
  WC_CUDA(cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking), detail);
  WC_TRY(put_csr(v.get(), v->fwd, csr->offsets, csr->targets, csr->weights, detail));
  v->host_offsets.assign(csr->offsets, csr->offsets + n + 1);
  // The reverse CSR: the caller's, or a transpose on the device.
  if (csr->reverse_offsets) {
    WC_TRY(put_csr(v.get(), v->rev, csr->reverse_offsets, csr->reverse_targets,
                   v->weighted ? csr->reverse_weights : nullptr, detail));
    v->host_rev_offsets.assign(csr->reverse_offsets, csr->reverse_offsets + n + 1);
    v->reverse_given = true;
  } else {
    WC_TRY(device_reverse(v.get(), detail));
    v->reverse_given = csr->reverse_on_device != 0;
  }
  WC_TRY(finish_version(v.get(), detail));
  *out = v.release();
  return WC_OK;
}

wc_status wc_version_release(wc_version* v) {
  if (!v || v->cursors.load() != 0) return WC_INVALID_ARGUMENT;
  {
    std::lock_guard<std::recursive_mutex> lock(v->mu);
    if (v->stream) cudaStreamSynchronize(v->stream);
    for (auto& g : v->graphs)
      if (g.second) cudaGraphExecDestroy(g.second);
    if (v->cancel_host) cudaFreeHost(v->cancel_host);
    if (v->stage_host) cudaFreeHost(v->stage_host);
    if (v->stream) cudaStreamDestroy(v->stream);
  }
  pagerank_part_forget(v);
  bfs_part_forget(v);
  delete v;
  return WC_OK;
}

wc_status wc_version_info_get(const wc_version* v, wc_version_info* info) {
  if (!v || !info) return WC_INVALID_ARGUMENT;
  info->id_space = v->n;
  info->edges = v->m;
  uint64_t bytes = 0;
  for (const DevCsr* d : {&v->fwd, &v->rev, &v->loc.csc})
    bytes += d->offsets.bytes + d->targets.bytes + d->weights.bytes + d->iweights.bytes +
             d->schedule.units.bytes + d->schedule.counters.bytes + d->schedule.carry.bytes +
             d->schedule.long_list.bytes + d->schedule.row_masks.bytes;
  bytes += v->loc.perm.bytes + v->loc.order.bytes;
  info->device_bytes = bytes;
  uint64_t pooled = 0;
  for (const auto& kv : v->pool) pooled += kv.second.bytes;
  info->scratch_bytes = pooled;
  info->weighted = v->weighted;
  info->integral_weights = v->integral;
  info->device = v->device;
  info->symmetric = v->symmetric;
  return WC_OK;
}

wc_status wc_version_sync(wc_version* v, const wc_call* call) {
  if (!v) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  Ctx ctx(v, call);
  return ctx.finish();
}

uint64_t wc_kernel_launches(void) { return g_launches.load(); }

double wc_version_timing(const wc_version* v, const char* phase, uint32_t* launches) {
  if (launches) *launches = 0;
  if (!v || !phase) return 0.0;
  auto it = v->timings.find(phase);
  if (it == v->timings.end()) return 0.0;
  if (launches) *launches = it->second.second;
  return it->second.first;
}

int32_t wc_serves(const char* op, wc_dtype dtype) {
  if (!op) return 0;
  std::string o(op);
  if (o == "spmv" || o == "spmm") return dtype >= WC_F32 && dtype <= WC_BOOL;
  if (o == "pagerank" || o == "eigen") return dtype == WC_F64;
  if (o == "bfs" || o == "reachable_set" || o == "reachable" || o == "components") return 1;
  if (o == "closeness_centrality" || o == "harmonic_centrality" || o == "betweenness_centrality")
    return dtype == WC_F64;
  if (o == "vector_reduce" || o == "vector_norm_diff" || o == "vector_map")
    return dtype >= WC_F32 && dtype <= WC_BOOL;
  if (o == "vector_topk") return dtype == WC_F64;
  return 0;
}

wc_status wc_host_transpose(uint64_t n, uint64_t m, const uint64_t* off, const uint32_t* tgt,
                            const double* w, uint64_t* roff, uint32_t* rtgt, double* rw) {
  if (!off || !roff || (m && (!tgt || !rtgt))) return WC_INVALID_ARGUMENT;
  host_transpose(n, m, off, tgt, w, roff, rtgt, rw);
  return WC_OK;
}

}  // extern "C"
