// components.cu — wc_components: weakly connected components,
// traversal/components.rs:21-58, each node labelled with the smallest dense
// id of its component.
//
// The reference unions the forward rows' edges in ascending order, always
// hanging the larger root under the smaller; the labels do not depend on
// the order, only on the components.  Here every edge hooks the larger of
// its two roots under the smaller with an atomic minimum (each node's parent
// stays at most the node, so every chain ends), then every node jumps to its
// root; rounds repeat until no edge joins two roots.  The roots are then the
// smallest ids of their components, as in the reference.
#include "operand.h"
#include "runtime.cuh"

namespace wc {

__global__ void wcc_init_kernel(uint32_t* parent, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    parent[i] = i;
}

// A warp per row; an edge whose endpoints have different roots hooks the
// larger root under the smaller.
__global__ void wcc_hook_kernel(const uint32_t* off, const uint32_t* tgt, uint32_t n,
                                uint32_t* parent, int* changed) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  bool hooked = false;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    const uint32_t lo = off[u], hi = off[u + 1];
    for (uint32_t e = lo + lane; e < hi; e += 32) {
      uint32_t a = parent[u], b = parent[tgt[e]];
      while (a != parent[a]) a = parent[a];  // parents only decrease: every chain ends
      while (b != parent[b]) b = parent[b];
      if (a != b) {
        atomicMin(parent + max(a, b), min(a, b));
        hooked = true;
      }
    }
  }
  // One write of the flag a warp (every edge writing it contended on one
  // address).
  if (__any_sync(0xffffffffu, hooked) && lane == 0) *changed = 1;
}

__global__ void wcc_compress_kernel(uint32_t* parent, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t r = parent[i];
    while (r != parent[r]) r = parent[r];
    parent[i] = r;
  }
}

__global__ void wcc_labels_kernel(const uint32_t* parent, uint32_t n, uint64_t* labels) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    labels[i] = parent[i];
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_components(wc_version* v, const wc_call* call, uint64_t* labels_out,
                        wc_traversal_stats* stats) {
  if (!v || (v->n && !labels_out)) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  const uint32_t n = (uint32_t)v->n;
  if (stats) *stats = wc_traversal_stats{n, v->m, 0, 0, 0};
  if (n == 0) return WC_OK;
  WC_TRY(ctx.begin());
  DevBuf *parent, *flag;
  WC_TRY(ctx.scratch(POOL_WCC_PARENT, (uint64_t)n * 4, &parent));
  WC_TRY(ctx.scratch(POOL_WCC_FLAG, 16, &flag));
  Operand L(POOL_WCC_LABELS);
  WC_TRY(L.output(ctx, labels_out, (uint64_t)n * 8));
  uint32_t* par = parent->as<uint32_t>();
  int* changed = flag->as<int>();
  const uint32_t grid = max_blocks(4);
  note_launch(), wcc_init_kernel<<<grid, 256, 0, ctx.stream>>>(par, n);
  // Each round at least halves the distance to the final roots; the bound
  // is far above what any graph needs.
  bool settled = false;
  for (int round = 0; round < 1000 && !settled; round++) {
    WC_CUDA(cudaMemsetAsync(changed, 0, 4, ctx.stream), ctx.detail);
    note_launch(), wcc_hook_kernel<<<max_blocks(8), 256, 0, ctx.stream>>>(
        v->fwd.offsets.as<uint32_t>(), v->fwd.targets.as<uint32_t>(), n, par, changed);
    note_launch(), wcc_compress_kernel<<<grid, 256, 0, ctx.stream>>>(par, n);
    int h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, changed, 4, cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
    WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
    if (ctx.cancelled()) return WC_CANCELLED;
    settled = h == 0;
  }
  if (!settled) return WC_DEVICE_TIMEOUT;
  note_launch(), wcc_labels_kernel<<<grid, 256, 0, ctx.stream>>>(par, n,
                                                                 static_cast<uint64_t*>(L.dev));
  WC_TRY(L.out(ctx));
  return ctx.finish();
}

}  // extern "C"
