// operand.h — a call's operand on the device: the caller's own device
// pointer, or a staging copy of a host buffer (copied in before the kernels
// and, for outputs, back out after them, on the call's stream).
#pragma once

#include "runtime.cuh"

namespace wc {

struct Operand {
  void* dev = nullptr;
  void* host_out = nullptr;
  bool is_device = true;
  uint64_t bytes = 0;
  int tag;

  explicit Operand(int pool_tag) : tag(pool_tag) {}

  wc_status stage(Ctx& ctx, const void* p, uint64_t n, bool copy_in) {
    bytes = n;
    if (is_device_pointer(p)) {
      dev = const_cast<void*>(p);
      is_device = true;
      return WC_OK;
    }
    is_device = false;
    DevBuf* staging;
    WC_TRY(ctx.scratch(tag, n, &staging));
    dev = staging->ptr;
    if (copy_in && n)
      WC_CUDA(cudaMemcpyAsync(dev, p, n, cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
    return WC_OK;
  }
  wc_status in(Ctx& ctx, const void* p, uint64_t n) { return stage(ctx, p, n, true); }
  wc_status inout(Ctx& ctx, void* p, uint64_t n) {
    host_out = p;
    return stage(ctx, p, n, true);
  }
  wc_status output(Ctx& ctx, void* p, uint64_t n) {
    host_out = p;
    return stage(ctx, p, n, false);
  }
  wc_status out(Ctx& ctx) {
    if (!is_device && host_out && bytes)
      WC_CUDA(cudaMemcpyAsync(host_out, dev, bytes, cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
    return WC_OK;
  }
};

// Helpers shared by the entry points (product.cu).
uint32_t max_blocks(int per_sm);
size_t dtype_size(int dtype);

}  // namespace wc
