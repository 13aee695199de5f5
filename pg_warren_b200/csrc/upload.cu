// upload.cu — a version's device copy built on the device: the reverse CSR
// by a device transpose, the weights' facts, the symmetry test, and the
// version loaded straight from its stored segments (graph/segment/csr.rs),
// checked on the device as Csr::from_segments checks them
// (graph/csr/mod.rs:78-137).
//
// The transpose sorts the forward entries by (target, source) — a 64-bit
// key, target in the high word — with the weights riding along; the radix
// sort is stable, so each reverse row comes out in ascending source order
// and duplicate entries keep their order, as the reference's counting
// transpose gives them (graph/csr/transpose.rs:14-44).
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include <cub/cub.cuh>

#include "operand.h"
#include "product.h"
#include "runtime.cuh"
#include "upload.h"

namespace wc {

// ------------------------------------------------------------ transpose

// The key of every forward entry: target << 32 | source.  A warp per row.
__global__ void transpose_keys_kernel(const uint32_t* off, const uint32_t* tgt, uint32_t n,
                                      uint64_t* keys) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps)
    for (uint32_t e = off[r] + lane; e < off[r + 1]; e += 32)
      keys[e] = ((uint64_t)tgt[e] << 32) | r;
}

// Reverse offsets from the sorted keys: entry e starts every row in
// (target(e - 1), target(e)]; the end m starts the rows after the last
// target.  Each offset is written once.
__global__ void reverse_offsets_kernel(const uint64_t* keys, uint64_t m, uint32_t n,
                                       uint32_t* roff) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e <= m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t hi = e < m ? (uint32_t)(keys[e] >> 32) : n;
    const uint32_t lo = e == 0 ? 0 : (uint32_t)(keys[e - 1] >> 32) + 1;
    for (uint32_t r = lo; r <= hi; r++) roff[r] = (uint32_t)e;
  }
}

__global__ void unpack_sources_kernel(const uint64_t* keys, uint64_t m, uint32_t* rtgt) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    rtgt[e] = (uint32_t)keys[e];
}

// ---------------------------------------------------------- weight facts

// Whether every weight is an integer in i32 range (an exact i32 copy is then
// kept) and the largest magnitude among them.
__global__ void weight_facts_kernel(const double* w, uint64_t m, unsigned* nonintegral,
                                    unsigned long long* max_abs) {
  unsigned long long mine = 0;
  int bad = 0;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const double x = w[e];
    const bool integral = x >= -2147483648.0 && x <= 2147483647.0 && x == (double)(int32_t)x;
    if (!integral) bad = 1;
    else mine = max(mine, (unsigned long long)llabs((long long)x));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mine = max(mine, __shfl_down_sync(0xffffffffu, mine, o));
    bad |= __shfl_down_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (bad) atomicOr(nonintegral, 1u);
    if (mine) atomicMax(max_abs, mine);
  }
}

__global__ void int_weights_kernel(const double* w, uint64_t m, int32_t* wi) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    wi[e] = (int32_t)w[e];
}

template <class T>
__global__ void differ_kernel(const T* a, const T* b, uint64_t len, unsigned* differ) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (!(a[i] == b[i])) {
      *differ = 1;
      return;
    }
}

static uint32_t grid_for(uint64_t items) {
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(max_blocks(8), (items + 255) / 256));
}

wc_status device_reverse(wc_version* v, wc_error_detail* detail) {
  const uint64_t n = v->n, m = v->m;
  cudaStream_t st = v->stream;
  DevCsr& f = v->fwd;
  DevCsr& r = v->rev;
  WC_TRY(r.offsets.alloc(v->budget, (n + 1) * 4 + kBulkPad, detail));
  WC_TRY(r.targets.alloc(v->budget, m * 4 + kBulkPad, detail));
  if (v->weighted) WC_TRY(r.weights.alloc(v->budget, m * 8 + kBulkPad, detail));
  v->host_rev_offsets.assign(n + 1, 0);
  if (m == 0) {
    WC_CUDA(cudaMemsetAsync(r.offsets.ptr, 0, (n + 1) * 4, st), detail);
    return cuda_status(cudaStreamSynchronize(st), detail, "reverse CSR");
  }
  DevBuf k0, k1, w0, w1, temp;
  WC_TRY(k0.alloc(v->budget, m * 8, detail));
  WC_TRY(k1.alloc(v->budget, m * 8, detail));
  note_launch(), transpose_keys_kernel<<<max_blocks(8), 256, 0, st>>>(
      f.offsets.as<uint32_t>(), f.targets.as<uint32_t>(), (uint32_t)n, k0.as<uint64_t>());
  // Sort on the source bits and the target's significant bits only.
  int target_bits = 1;
  while (target_bits < 32 && (1ull << target_bits) < n) target_bits++;
  const int end_bit = 32 + target_bits;
  cub::DoubleBuffer<uint64_t> keys(k0.as<uint64_t>(), k1.as<uint64_t>());
  size_t temp_bytes = 0;
  if (v->weighted) {
    WC_TRY(w0.alloc(v->budget, m * 8, detail));
    WC_TRY(w1.alloc(v->budget, m * 8, detail));
    WC_CUDA(cudaMemcpyAsync(w0.ptr, f.weights.ptr, m * 8, cudaMemcpyDeviceToDevice, st), detail);
    cub::DoubleBuffer<double> vals(w0.as<double>(), w1.as<double>());
    WC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, vals, m, 0, end_bit, st),
            detail);
    WC_TRY(temp.alloc(v->budget, std::max<size_t>(temp_bytes, 16), detail));
    WC_CUDA(cub::DeviceRadixSort::SortPairs(temp.ptr, temp_bytes, keys, vals, m, 0, end_bit, st),
            detail);
    WC_CUDA(cudaMemcpyAsync(r.weights.ptr, vals.Current(), m * 8, cudaMemcpyDeviceToDevice, st),
            detail);
  } else {
    WC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, keys, m, 0, end_bit, st), detail);
    WC_TRY(temp.alloc(v->budget, std::max<size_t>(temp_bytes, 16), detail));
    WC_CUDA(cub::DeviceRadixSort::SortKeys(temp.ptr, temp_bytes, keys, m, 0, end_bit, st), detail);
  }
  note_launch(), unpack_sources_kernel<<<grid_for(m), 256, 0, st>>>(keys.Current(), m,
                                                                   r.targets.as<uint32_t>());
  note_launch(), reverse_offsets_kernel<<<grid_for(m + 1), 256, 0, st>>>(
      keys.Current(), m, (uint32_t)n, r.offsets.as<uint32_t>());
  std::vector<uint32_t> roff(n + 1);
  WC_CUDA(cudaMemcpyAsync(roff.data(), r.offsets.ptr, (n + 1) * 4, cudaMemcpyDeviceToHost, st),
          detail);
  WC_CUDA(cudaStreamSynchronize(st), detail);
  for (uint64_t i = 0; i <= n; i++) v->host_rev_offsets[i] = roff[i];
  return WC_OK;
}

wc_status device_weight_facts(wc_version* v, wc_error_detail* detail) {
  v->integral = false;
  v->max_abs_iweight = 1;
  if (!v->weighted) return WC_OK;
  cudaStream_t st = v->stream;
  DevBuf flags;
  WC_TRY(flags.alloc(v->budget, 16, detail));
  WC_CUDA(cudaMemsetAsync(flags.ptr, 0, 16, st), detail);
  unsigned* nonintegral = flags.as<unsigned>();
  unsigned long long* max_abs =
      reinterpret_cast<unsigned long long*>(flags.as<unsigned char>() + 8);
  if (v->m)
    note_launch(), weight_facts_kernel<<<grid_for(v->m), 256, 0, st>>>(
        v->fwd.weights.as<double>(), v->m, nonintegral, max_abs);
  uint64_t host[2] = {0, 0};
  WC_CUDA(cudaMemcpyAsync(host, flags.ptr, 16, cudaMemcpyDeviceToHost, st), detail);
  WC_CUDA(cudaStreamSynchronize(st), detail);
  v->integral = (host[0] & 0xffffffffu) == 0;
  v->max_abs_iweight = v->integral ? (int64_t)host[1] : -1;
  if (!v->integral) return WC_OK;
  for (DevCsr* d : {&v->fwd, &v->rev}) {
    WC_TRY(d->iweights.alloc(v->budget, v->m * 4 + kBulkPad, detail));
    if (v->m)
      note_launch(), int_weights_kernel<<<grid_for(v->m), 256, 0, st>>>(
          d->weights.as<double>(), v->m, d->iweights.as<int32_t>());
  }
  return cuda_status(cudaStreamSynchronize(st), detail, "integral weights");
}

wc_status device_symmetric(wc_version* v, wc_error_detail* detail) {
  cudaStream_t st = v->stream;
  DevBuf flag;
  WC_TRY(flag.alloc(v->budget, 4, detail));
  WC_CUDA(cudaMemsetAsync(flag.ptr, 0, 4, st), detail);
  unsigned* d = flag.as<unsigned>();
  note_launch(), differ_kernel<uint32_t><<<grid_for(v->n + 1), 256, 0, st>>>(
      v->fwd.offsets.as<uint32_t>(), v->rev.offsets.as<uint32_t>(), v->n + 1, d);
  if (v->m) {
    note_launch(), differ_kernel<uint32_t><<<grid_for(v->m), 256, 0, st>>>(
        v->fwd.targets.as<uint32_t>(), v->rev.targets.as<uint32_t>(), v->m, d);
    if (v->weighted)
      note_launch(), differ_kernel<double><<<grid_for(v->m), 256, 0, st>>>(
          v->fwd.weights.as<double>(), v->rev.weights.as<double>(), v->m, d);
  }
  unsigned differ = 0;
  WC_CUDA(cudaMemcpyAsync(&differ, d, 4, cudaMemcpyDeviceToHost, st), detail);
  WC_CUDA(cudaStreamSynchronize(st), detail);
  v->symmetric = differ == 0;
  return WC_OK;
}

// -------------------------------------------------------------- segments

constexpr uint64_t kNone = ~0ull;

// Stored rows (sparse offsets): the first position j >= 1 not above the
// row before it, and the first stored row without targets.
__global__ void stored_rows_kernel(const uint32_t* rows, const uint64_t* off, uint64_t count,
                                   unsigned long long* first) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count;
       j += (uint64_t)gridDim.x * blockDim.x) {
    if (j && rows[j] <= rows[j - 1]) atomicMin(first, (unsigned long long)j);
    if (off[j + 1] <= off[j]) atomicMin(first + 1, (unsigned long long)j);
  }
}

// The first position whose next offset is smaller.
__global__ void monotone_kernel(const uint64_t* off, uint64_t count, unsigned long long* first) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < count;
       p += (uint64_t)gridDim.x * blockDim.x)
    if (off[p + 1] < off[p]) atomicMin(first, (unsigned long long)p);
}

// Per stored position p (a warp each, offsets already monotone and ending
// at m): 2p if the row has a target outside the id space, else 2p + 1 if
// it is not strictly ascending; the minimum over the rows.
__global__ void row_targets_kernel(const uint64_t* off, uint64_t count, const uint32_t* tgt,
                                   uint64_t n, unsigned long long* first) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < count;
       p += warps) {
    bool outside = false, unsorted = false;
    for (uint64_t e = off[p] + lane; e < off[p + 1]; e += 32) {
      const uint32_t t = tgt[e];
      outside |= t >= n;
      unsorted |= e > off[p] && tgt[e - 1] >= t;
    }
    outside = __any_sync(0xffffffffu, outside);
    unsorted = __any_sync(0xffffffffu, unsorted);
    if (lane == 0 && (outside || unsorted))
      atomicMin(first, (unsigned long long)(2 * p + (outside ? 0 : 1)));
  }
}

// Dense u32 offsets over the id space: node i starts at the offset of the
// first stored row at or after it (the end m past the last).
__global__ void dense_offsets_kernel(const uint32_t* rows, const uint64_t* off, uint64_t count,
                                     uint32_t n, uint32_t* dense) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = i;
    if (rows) {
      uint64_t lo = 0, hi = count;  // lower_bound(rows, i)
      while (lo < hi) {
        const uint64_t mid = (lo + hi) / 2;
        if (rows[mid] < i) lo = mid + 1;
        else hi = mid;
      }
      j = lo;
    }
    dense[i] = (uint32_t)off[j];
  }
}

struct Segment {
  const uint8_t* payload = nullptr;
  uint64_t payload_len = 0, count = 0;
  uint8_t width = 0;
};

static uint64_t le64(const uint8_t* p) {
  uint64_t x = 0;
  for (int b = 7; b >= 0; b--) x = (x << 8) | p[b];
  return x;
}
static uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// segment/mod.rs:276-296 (read_header): the header's checks in order.
static wc_status read_header(const uint8_t* bytes, uint64_t len, uint8_t kind, Segment* s,
                             wc_error_detail* d) {
  if (!bytes || len < 16) {
    set_message(d, "segment truncated");
    return WC_SEGMENT_TRUNCATED;
  }
  if (std::memcmp(bytes, "WRSG", 4) != 0) {
    set_message(d, "not a pg_warren segment");
    return WC_SEGMENT_MAGIC;
  }
  if (bytes[4] != 2) {  // a CSR's segments are format 2 (segment/mod.rs:35-43)
    if (d) d->found = bytes[4];
    set_message(d, "unsupported segment format %u: a version built by an earlier pg_warren must "
                   "be built again with warren.refresh", bytes[4]);
    return WC_SEGMENT_FORMAT;
  }
  if (bytes[5] != kind) {
    if (d) d->expected = kind, d->found = bytes[5];
    set_message(d, "segment kind %u, expected %u", bytes[5], kind);
    return WC_SEGMENT_KIND;
  }
  if (bytes[7] != 0) {
    if (d) d->found = bytes[7];
    set_message(d, "segment reserved byte is %u, expected 0", bytes[7]);
    return WC_SEGMENT_RESERVED;
  }
  s->width = bytes[6];
  s->count = le64(bytes + 8);
  s->payload = bytes + 16;
  s->payload_len = len - 16;
  return WC_OK;
}

// segment/mod.rs:299-322 (expect_width, expect_length).
static wc_status check_elements(const Segment& s, uint8_t width, wc_error_detail* d) {
  if (s.width != width) {
    if (d) d->expected = width, d->found = s.width;
    set_message(d, "segment element width %u, expected %u", s.width, width);
    return WC_SEGMENT_WIDTH;
  }
  const unsigned __int128 expected = (unsigned __int128)s.count * width;
  if (expected != s.payload_len) {
    const uint64_t e = expected > ~0ull ? ~0ull : (uint64_t)expected;
    if (d) d->expected = e, d->found = s.payload_len;
    set_message(d, "segment payload is %llu, expected %llu", (unsigned long long)s.payload_len,
                (unsigned long long)e);
    return WC_SEGMENT_LENGTH;
  }
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_version_load_segments(uint64_t graph_id, uint64_t version, uint64_t id_space,
                                   const uint8_t* rows_segment, uint64_t rows_len,
                                   const uint8_t* offsets_segment, uint64_t offsets_len,
                                   const uint8_t* targets_segment, uint64_t targets_len,
                                   const uint8_t* weights_segment, uint64_t weights_len,
                                   int32_t has_reverse, wc_budget* budget, const wc_call* call,
                                   wc_version** out) {
  wc_error_detail* d = call ? call->detail : nullptr;
  if (!out) return WC_INVALID_ARGUMENT;
  *out = nullptr;
  // AnyCsr::decode (segment/csr.rs:83-122): offsets, weights, the rows'
  // and targets' headers, then the targets' and rows' elements.
  Segment off, tg, rw, wt;
  WC_TRY(read_header(offsets_segment, offsets_len, 1, &off, d));
  WC_TRY(check_elements(off, 8, d));
  if (weights_segment) {
    WC_TRY(read_header(weights_segment, weights_len, 3, &wt, d));
    WC_TRY(check_elements(wt, 8, d));
  }
  if (rows_segment) WC_TRY(read_header(rows_segment, rows_len, 11, &rw, d));
  WC_TRY(read_header(targets_segment, targets_len, 2, &tg, d));
  if (id_space >= (1ull << 32) || tg.count >= (1ull << 32)) {
    set_message(d, "id spaces and edge counts of 2^32 or more are not served");
    return WC_UNSUPPORTED;
  }
  WC_TRY(check_elements(tg, 4, d));
  if (rows_segment) WC_TRY(check_elements(rw, 4, d));
  // Csr::from_segments (graph/csr/mod.rs:78-137): on the host where one
  // element decides, on the device where every element must be read.
  const uint64_t n = id_space, m = tg.count;
  const uint64_t stored = rows_segment ? rw.count : n;
  if (off.count != stored + 1) {
    if (d) d->expected = stored + 1, d->found = off.count;
    set_message(d, "CSR has %llu offsets, expected %llu", (unsigned long long)off.count,
                (unsigned long long)(stored + 1));
    return WC_OFFSETS_LENGTH;
  }
  if (le64(off.payload) != 0) {
    set_message(d, "CSR offsets do not start at 0");
    return WC_FIRST_OFFSET_NOT_ZERO;
  }
  WC_TRY(wc_device_check(d));
  std::unique_ptr<wc_version> v(new wc_version);
  v->graph_id = graph_id;
  v->version = version;
  v->n = n;
  v->m = m;
  v->budget = budget;
  v->budget_ref.hold(budget);
  v->weighted = weights_segment != nullptr;
  WC_CUDA(cudaGetDevice(&v->device), d);
  WC_CUDA(cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking), d);
  cudaStream_t st = v->stream;
  DevBuf doff, drows, first;
  WC_TRY(doff.alloc(budget, (stored + 1) * 8, d));
  WC_CUDA(cudaMemcpyAsync(doff.ptr, off.payload, (stored + 1) * 8, cudaMemcpyHostToDevice, st), d);
  const uint32_t* rows_dev = nullptr;
  if (rows_segment) {
    WC_TRY(drows.alloc(budget, std::max<uint64_t>(stored * 4, 4), d));
    if (stored)
      WC_CUDA(cudaMemcpyAsync(drows.ptr, rw.payload, stored * 4, cudaMemcpyHostToDevice, st), d);
    rows_dev = drows.as<uint32_t>();
  }
  WC_TRY(v->fwd.targets.alloc(budget, m * 4 + kBulkPad, d));
  if (m)
    WC_CUDA(cudaMemcpyAsync(v->fwd.targets.ptr, tg.payload, m * 4, cudaMemcpyHostToDevice, st), d);
  WC_TRY(first.alloc(budget, 32, d));
  unsigned long long* fw = first.as<unsigned long long>();
  uint64_t host[4];
  auto firsts = [&]() -> wc_status {
    WC_CUDA(cudaMemcpyAsync(host, fw, 32, cudaMemcpyDeviceToHost, st), d);
    return cuda_status(cudaStreamSynchronize(st), d, "segment checks");
  };
  const uint64_t* off_dev = doff.as<uint64_t>();
  auto row_id = [&](uint64_t p) -> uint64_t {
    return rows_segment ? le32(rw.payload + 4 * p) : p;
  };
  if (rows_segment) {  // check_stored_rows (csr/mod.rs:241-258)
    WC_CUDA(cudaMemsetAsync(fw, 0xff, 32, st), d);
    if (stored)
      note_launch(), stored_rows_kernel<<<grid_for(stored), 256, 0, st>>>(rows_dev, off_dev,
                                                                        stored, fw);
    WC_TRY(firsts());
    if (host[0] != kNone) {
      if (d) d->node = host[0];
      set_message(d, "CSR stored row %llu is not above the one before it",
                  (unsigned long long)host[0]);
      return WC_STORED_ROWS_NOT_ASCENDING;
    }
    if (stored && row_id(stored - 1) >= n) {
      if (d) d->node = row_id(stored - 1);
      set_message(d, "CSR stores row %llu, outside the id space",
                  (unsigned long long)row_id(stored - 1));
      return WC_STORED_ROW_OUTSIDE_ID_SPACE;
    }
    if (host[1] != kNone) {
      if (d) d->node = row_id(host[1]);
      set_message(d, "CSR stores row %llu without targets", (unsigned long long)row_id(host[1]));
      return WC_STORED_ROW_EMPTY;
    }
  }
  WC_CUDA(cudaMemsetAsync(fw, 0xff, 32, st), d);
  if (stored)
    note_launch(), monotone_kernel<<<grid_for(stored), 256, 0, st>>>(off_dev, stored, fw);
  WC_TRY(firsts());
  if (host[0] != kNone) {
    if (d) d->node = row_id(host[0]);
    set_message(d, "CSR offsets decrease after row %llu", (unsigned long long)row_id(host[0]));
    return WC_OFFSETS_NOT_MONOTONE;
  }
  const uint64_t last = le64(off.payload + 8 * stored);
  if (last != m) {
    if (d) d->expected = m, d->found = last;
    set_message(d, "CSR final offset is %llu, expected %llu", (unsigned long long)last,
                (unsigned long long)m);
    return WC_FINAL_OFFSET;
  }
  WC_CUDA(cudaMemsetAsync(fw, 0xff, 32, st), d);
  if (stored)
    note_launch(), row_targets_kernel<<<max_blocks(8), 256, 0, st>>>(
        off_dev, stored, v->fwd.targets.as<uint32_t>(), n, fw);
  WC_TRY(firsts());
  if (host[0] != kNone) {
    const uint64_t p = host[0] / 2, row = row_id(p);
    if (d) d->node = row;
    if (host[0] % 2 == 0) {
      uint64_t target = 0;
      for (uint64_t e = le64(off.payload + 8 * p); e < le64(off.payload + 8 * (p + 1)); e++)
        if ((target = le32(tg.payload + 4 * e)) >= n) break;
      if (d) d->found = target;
      set_message(d, "CSR row %llu has target %llu outside the id space", (unsigned long long)row,
                  (unsigned long long)target);
      return WC_TARGET_OUTSIDE_ID_SPACE;
    }
    set_message(d, "CSR row %llu is not strictly ascending", (unsigned long long)row);
    return WC_ROW_NOT_SORTED;
  }
  if (weights_segment && wt.count != m) {
    if (d) d->expected = m, d->found = wt.count;
    set_message(d, "CSR has %llu weights, expected %llu", (unsigned long long)wt.count,
                (unsigned long long)m);
    return WC_WEIGHTS_LENGTH;
  }
  // The device copy: dense u32 offsets and the weights, then what every
  // version gets.
  WC_TRY(v->fwd.offsets.alloc(budget, (n + 1) * 4 + kBulkPad, d));
  note_launch(), dense_offsets_kernel<<<grid_for(n + 1), 256, 0, st>>>(
      rows_dev, off_dev, stored, (uint32_t)n, v->fwd.offsets.as<uint32_t>());
  if (v->weighted) {
    WC_TRY(v->fwd.weights.alloc(budget, m * 8 + kBulkPad, d));
    if (m)
      WC_CUDA(cudaMemcpyAsync(v->fwd.weights.ptr, wt.payload, m * 8, cudaMemcpyHostToDevice, st),
              d);
  }
  std::vector<uint32_t> dense(n + 1);
  WC_CUDA(cudaMemcpyAsync(dense.data(), v->fwd.offsets.ptr, (n + 1) * 4, cudaMemcpyDeviceToHost,
                          st), d);
  WC_CUDA(cudaStreamSynchronize(st), d);
  v->host_offsets.assign(dense.begin(), dense.end());
  doff.release();
  drows.release();
  first.release();
  WC_TRY(device_reverse(v.get(), d));
  v->reverse_given = has_reverse != 0;
  WC_TRY(finish_version(v.get(), d));
  *out = v.release();
  return WC_OK;
}

}  // extern "C"
