// product.cu — wc_spmv / wc_spmm: compute/product/mod.rs:77-205 on the
// device.  Aᵀ is always pulled over the device's reverse CSR; the reference
// pushes only where it has no reverse CSR, and its push and pull agree bit
// for bit (product/mod.rs:8-12), so the result is the same.
#include <algorithm>
#include <vector>

#include "operand.h"
#include "product.h"
#include "semiring.cuh"

namespace wc {

uint32_t max_blocks(int per_sm) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return (uint32_t)(sms * per_sm);
}

size_t dtype_size(int dtype) {
  switch (dtype) {
    case WC_F64: case WC_I64: return 8;
    case WC_F32: return 4;
    default: return 1;
  }
}

// Fills a launch description for `csr` and the product.
wc_status prepare_pull(Ctx& ctx, DevCsr& csr, int semiring, int weighted_flag, int dtype,
                       uint32_t width, PullLaunch& L) {
  wc_version* v = ctx.v;
  bool weighted = weighted_flag != 0 && v->weighted;
  L = PullLaunch{};
  L.off = csr.offsets.as<uint32_t>();
  L.tgt = csr.targets.as<uint32_t>();
  L.weight_kind = WEIGHTS_NONE;
  L.weights = nullptr;
  if (weighted) {
    // The int32 copy is exact for every element type whose cast of an
    // integral weight is the integer itself (i64); others read the f64.
    if (dtype == WC_I64 && v->integral) {
      L.weight_kind = WEIGHTS_I32;
      L.weights = csr.iweights.ptr;
    } else {
      L.weight_kind = WEIGHTS_F64;
      L.weights = csr.weights.ptr;
    }
  }
  L.units = csr.schedule.units.as<Unit>();
  L.unit_count = csr.schedule.count;
  L.counters = csr.schedule.counters.as<uint32_t>();
  L.carry = csr.schedule.carry.ptr;
  L.n = (uint32_t)v->n;
  L.width = width;
  L.semiring = semiring;
  L.max_blocks = max_blocks(8);
  L.stream = ctx.stream;
  L.err = v->error.as<DeviceError>();
  L.detail = ctx.detail;
  L.write = WriteArgs{nullptr, WC_F64, 0, 0, -1};
  return WC_OK;
}

wc_status launch_pull(const PullLaunch& L, int dtype, const void* x, void* y) {
  switch (dtype) {
    case WC_F64: return launch_pull_f64(L, x, y);
    case WC_F32: return launch_pull_f32(L, x, y);
    case WC_I64: return launch_pull_i64(L, x, y);
    case WC_BOOL: return launch_pull_bool(L, x, y);
  }
  return WC_DTYPE_MISMATCH;
}

// `parts` > 0: only part `part` of the rows (schedule_part_cuts over the
// product's CSR) is computed and written; y's other rows are left as given.
static wc_status product(wc_version* v, const wc_call* call, const wc_product* p, wc_dtype dtype,
                         uint32_t width, const void* x, void* y, uint32_t parts = 0,
                         uint32_t part = 0) {
  if (!v || !p || !x || !y) return WC_INVALID_ARGUMENT;
  if (parts && part >= parts) return WC_INVALID_ARGUMENT;
  if (p->semiring < 0 || p->semiring > WC_MAX_SECOND) return WC_UNKNOWN_SEMIRING;
  if (dtype < WC_F32 || dtype > WC_BOOL) return WC_DTYPE_MISMATCH;
  if (width == 0) return WC_ZERO_WIDTH;
  if (p->accumulate != WC_OP_NONE && (p->accumulate < WC_OP_FIRST || p->accumulate > WC_OP_ANY))
    return WC_UNKNOWN_BINARY_OP;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  const size_t es = dtype_size(dtype);
  const uint64_t bytes = v->n * (uint64_t)width * es;
  Operand X(POOL_X), Y(POOL_Y), M(POOL_MASK);
  WC_TRY(X.in(ctx, x, bytes));
  WC_TRY(Y.inout(ctx, y, bytes));
  if (p->mask) {
    if (!p->mask->values) return WC_INVALID_ARGUMENT;
    WC_TRY(M.in(ctx, p->mask->values, v->n * dtype_size(p->mask->dtype)));
  }
  // x and y must not alias: the reference borrows them apart.
  const void* xd = X.dev;
  if (X.dev == Y.dev) {
    DevBuf* xcopy;
    WC_TRY(ctx.scratch(POOL_XCOPY, bytes, &xcopy));
    WC_CUDA(cudaMemcpyAsync(xcopy->ptr, X.dev, bytes, cudaMemcpyDeviceToDevice, ctx.stream),
            ctx.detail);
    xd = xcopy->ptr;
  }
  WC_TRY(ctx.begin());
  PullLaunch L;
  DevCsr& csr = p->transpose ? v->rev : v->fwd;
  WC_TRY(prepare_pull(ctx, csr, p->semiring, p->weighted, dtype, width, L));
  if (parts) {
    std::vector<uint32_t> uc;
    std::vector<uint64_t> rc;
    WC_TRY(schedule_part_cuts(v, csr, parts, uc, rc, ctx.detail));
    L.units += uc[part];
    L.unit_count = uc[part + 1] - uc[part];
  }
  if (width > 1) {
    DevBuf* mc;
    WC_TRY(ctx.scratch(POOL_SPMM_CARRY,
                       (uint64_t)std::max<uint32_t>(csr.schedule.slots, 1) * kMultiCarryBytesPerSlot,
                       &mc));
    L.carry_multi = mc->ptr;
  }
  if (p->mask) L.write = WriteArgs{M.dev, (int32_t)p->mask->dtype, p->mask->complement, p->replace,
                                   (int32_t)p->accumulate};
  else L.write = WriteArgs{nullptr, WC_F64, 0, p->replace, (int32_t)p->accumulate};
  if (L.unit_count) WC_TRY(launch_pull(L, dtype, xd, Y.dev));
  WC_TRY(Y.out(ctx));
  // Asynchronous only where every operand is the caller's device memory.
  if (ctx.async && X.is_device && Y.is_device && (!p->mask || M.is_device)) return WC_OK;
  return ctx.finish();
}

}  // namespace wc

extern "C" {

wc_status wc_spmv(wc_version* v, const wc_call* call, const wc_product* p, wc_dtype dtype,
                  const void* x, void* y) {
  return wc::product(v, call, p, dtype, 1, x, y);
}

wc_status wc_spmm(wc_version* v, const wc_call* call, const wc_product* p, wc_dtype dtype,
                  uint32_t width, const void* x, void* y) {
  return wc::product(v, call, p, dtype, width, x, y);
}

wc_status wc_spmv_part_rows(wc_version* v, int32_t transpose, uint32_t parts,
                            uint64_t* row_bounds) {
  if (!v || parts == 0 || !row_bounds) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), nullptr);
  std::vector<uint32_t> uc;
  std::vector<uint64_t> rc;
  WC_TRY(wc::schedule_part_cuts(v, transpose ? v->rev : v->fwd, parts, uc, rc, nullptr));
  std::copy(rc.begin(), rc.end(), row_bounds);
  return WC_OK;
}

wc_status wc_spmv_part(wc_version* v, const wc_call* call, const wc_product* p, wc_dtype dtype,
                       uint32_t parts, uint32_t part, const void* x, void* y) {
  if (parts == 0) return WC_INVALID_ARGUMENT;
  return wc::product(v, call, p, dtype, 1, x, y, parts, part);
}

}  // extern "C"
