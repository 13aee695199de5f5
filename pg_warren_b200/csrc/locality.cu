// locality.cu — a version's reverse CSR in locality order, for the pull
// solvers whose cost is the gather of x over the entries (PageRank).
//
// The nodes are renumbered by out-degree, largest first (equal degrees in
// dense-id order).  A pull over the reverse CSR reads x_j once per out-edge
// of j, so the nodes gathered most often get the lowest numbers: their
// values share 32-byte sectors and cache lines, and the most gathered of
// them stay in each SM's L1.  Row k of the renumbered CSC is the reverse row
// of node order[k] with its entries in their stored order and each source
// renumbered perm[source]; a row's fold adds the same products in the same
// order as over the plain CSC, so each row's result is the same bit for
// bit.  A solver keeps its per-node vectors in the new numbering and
// renumbers only at the boundary: inputs scattered in, results gathered out.
// (The reference's own locality orders, graph/node_order/, renumber the
// stored graph; this one is internal to the device copy.)
#include <algorithm>
#include <vector>

#include <cub/cub.cuh>

#include "operand.h"
#include "runtime.cuh"
#include "upload.h"

namespace wc {

__global__ void degree_keys_kernel(const uint32_t* fwd_off, uint32_t n, uint32_t* keys,
                                   uint32_t* ids) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = ~(fwd_off[i + 1] - fwd_off[i]);  // ascending keys: largest degree first
    ids[i] = i;
  }
}

__global__ void invert_kernel(const uint32_t* order, uint32_t n, uint32_t* perm) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    perm[order[k]] = k;
}

// New row k's entry count (the last slot, n, is zero for the scan).
__global__ void loc_degrees_kernel(const uint32_t* order, const uint32_t* roff, uint32_t n,
                                   uint32_t* deg) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x)
    deg[k] = k < n ? roff[order[k] + 1] - roff[order[k]] : 0u;
}

// A warp per new row: the old row's entries in order, sources renumbered.
__global__ void loc_entries_kernel(const uint32_t* order, const uint32_t* perm,
                                   const uint32_t* roff, const uint32_t* rtgt, const double* rw,
                                   const int32_t* rwi, const uint32_t* noff, uint32_t n,
                                   uint32_t* ntgt, double* nw, int32_t* nwi) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += warps) {
    const uint32_t r = order[k], a = roff[r], b = roff[r + 1], dst = noff[k];
    for (uint32_t e = a + lane; e < b; e += 32) {
      ntgt[dst + (e - a)] = perm[rtgt[e]];
      if (rw) nw[dst + (e - a)] = rw[e];
      if (rwi) nwi[dst + (e - a)] = rwi[e];
    }
  }
}

static uint32_t grid_of(uint64_t items) {
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(max_blocks(8), (items + 255) / 256));
}

wc_status device_locality(wc_version* v, wc_error_detail* detail) {
  const uint64_t n = v->n, m = v->m;
  cudaStream_t st = v->stream;
  Locality& L = v->loc;
  DevCsr& c = L.csc;
  WC_TRY(L.order.alloc(v->budget, std::max<uint64_t>(n, 1) * 4, detail));
  WC_TRY(L.perm.alloc(v->budget, std::max<uint64_t>(n, 1) * 4, detail));
  WC_TRY(c.offsets.alloc(v->budget, (n + 1) * 4 + kBulkPad, detail));
  WC_TRY(c.targets.alloc(v->budget, m * 4 + kBulkPad, detail));
  if (v->weighted) WC_TRY(c.weights.alloc(v->budget, m * 8 + kBulkPad, detail));
  if (v->weighted && v->integral) WC_TRY(c.iweights.alloc(v->budget, m * 4 + kBulkPad, detail));
  if (n) {
    // Order: a stable radix sort of (¬out-degree, id).
    DevBuf k0, k1, i1, temp;
    WC_TRY(k0.alloc(v->budget, n * 4, detail));
    WC_TRY(k1.alloc(v->budget, n * 4, detail));
    WC_TRY(i1.alloc(v->budget, n * 4, detail));
    note_launch(), degree_keys_kernel<<<grid_of(n), 256, 0, st>>>(
        v->fwd.offsets.as<uint32_t>(), (uint32_t)n, k0.as<uint32_t>(), L.order.as<uint32_t>());
    cub::DoubleBuffer<uint32_t> keys(k0.as<uint32_t>(), k1.as<uint32_t>());
    cub::DoubleBuffer<uint32_t> ids(L.order.as<uint32_t>(), i1.as<uint32_t>());
    size_t temp_bytes = 0;
    WC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, ids, (int)n, 0, 32, st),
            detail);
    WC_TRY(temp.alloc(v->budget, std::max<size_t>(temp_bytes, 16), detail));
    WC_CUDA(cub::DeviceRadixSort::SortPairs(temp.ptr, temp_bytes, keys, ids, (int)n, 0, 32, st),
            detail);
    if (ids.Current() != L.order.as<uint32_t>())
      WC_CUDA(cudaMemcpyAsync(L.order.ptr, ids.Current(), n * 4, cudaMemcpyDeviceToDevice, st),
              detail);
    note_launch(), invert_kernel<<<grid_of(n), 256, 0, st>>>(L.order.as<uint32_t>(), (uint32_t)n,
                                                              L.perm.as<uint32_t>());
    // Offsets: the new rows' entry counts, scanned (k1 holds the counts).
    DevBuf counts;
    WC_TRY(counts.alloc(v->budget, (n + 1) * 4, detail));
    note_launch(), loc_degrees_kernel<<<grid_of(n + 1), 256, 0, st>>>(
        L.order.as<uint32_t>(), v->rev.offsets.as<uint32_t>(), (uint32_t)n, counts.as<uint32_t>());
    size_t scan_bytes = 0;
    WC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts.as<uint32_t>(),
                                          c.offsets.as<uint32_t>(), (int)(n + 1), st),
            detail);
    if (scan_bytes > temp.bytes) WC_TRY(temp.alloc(v->budget, scan_bytes, detail));
    WC_CUDA(cub::DeviceScan::ExclusiveSum(temp.ptr, scan_bytes, counts.as<uint32_t>(),
                                          c.offsets.as<uint32_t>(), (int)(n + 1), st),
            detail);
    if (m)
      note_launch(), loc_entries_kernel<<<max_blocks(8), 256, 0, st>>>(
          L.order.as<uint32_t>(), L.perm.as<uint32_t>(), v->rev.offsets.as<uint32_t>(),
          v->rev.targets.as<uint32_t>(), v->weighted ? v->rev.weights.as<double>() : nullptr,
          c.iweights.ptr ? v->rev.iweights.as<int32_t>() : nullptr, c.offsets.as<uint32_t>(),
          (uint32_t)n, c.targets.as<uint32_t>(), c.weights.as<double>(), c.iweights.as<int32_t>());
    WC_CUDA(cudaStreamSynchronize(st), detail);  // before the transient buffers go
  } else {
    WC_CUDA(cudaMemsetAsync(c.offsets.ptr, 0, 4, st), detail);
  }
  std::vector<uint32_t> off32(n + 1);
  WC_CUDA(cudaMemcpyAsync(off32.data(), c.offsets.ptr, (n + 1) * 4, cudaMemcpyDeviceToHost, st),
          detail);
  WC_CUDA(cudaStreamSynchronize(st), detail);
  std::vector<uint64_t> off(off32.begin(), off32.end());
  WC_TRY(put_schedule(v, c, off, detail));
  return cuda_status(cudaGetLastError(), detail, "locality order");
}

// ------------------------------------------------- renumbering vectors

__global__ void scatter_f64_kernel(const double* src, const uint32_t* perm, uint32_t n,
                                   double* dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[perm[i]] = src[i];
}

__global__ void gather_f64_kernel(const double* src, const uint32_t* perm, uint32_t n,
                                  double* dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

__global__ void scatter_bits_kernel(const uint64_t* bits, const uint32_t* perm, uint32_t n,
                                    uint64_t* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if ((bits[i >> 6] >> (i & 63)) & 1) {
      const uint32_t k = perm[i];
      atomicOr(reinterpret_cast<unsigned long long*>(out + (k >> 6)), 1ull << (k & 63));
    }
}

wc_status to_locality(const wc_version* v, cudaStream_t st, const double* src, double* dst) {
  if (v->n)
    note_launch(), scatter_f64_kernel<<<grid_of(v->n), 256, 0, st>>>(
        src, v->loc.perm.as<uint32_t>(), (uint32_t)v->n, dst);
  return cuda_status(cudaGetLastError(), nullptr, "renumber in");
}

wc_status from_locality(const wc_version* v, cudaStream_t st, const double* src, double* dst) {
  if (v->n)
    note_launch(), gather_f64_kernel<<<grid_of(v->n), 256, 0, st>>>(
        src, v->loc.perm.as<uint32_t>(), (uint32_t)v->n, dst);
  return cuda_status(cudaGetLastError(), nullptr, "renumber out");
}

wc_status bits_to_locality(const wc_version* v, cudaStream_t st, const uint64_t* src,
                           uint64_t* dst) {
  const uint64_t words = (v->n + 63) / 64;
  WC_CUDA(cudaMemsetAsync(dst, 0, words * 8, st), nullptr);
  if (v->n)
    note_launch(), scatter_bits_kernel<<<grid_of(v->n), 256, 0, st>>>(
        src, v->loc.perm.as<uint32_t>(), (uint32_t)v->n, dst);
  return cuda_status(cudaGetLastError(), nullptr, "renumber bits");
}

wc_status locality_status(Ctx& ctx, wc_status st) {
  if (st == WC_OK || !ctx.device_error || !ctx.detail || ctx.detail->node >= ctx.v->n) return st;
  uint32_t id = 0;
  if (cudaMemcpy(&id, ctx.v->loc.order.as<uint32_t>() + ctx.detail->node, 4,
                 cudaMemcpyDeviceToHost) == cudaSuccess)
    ctx.detail->node = id;
  return st;
}

}  // namespace wc
