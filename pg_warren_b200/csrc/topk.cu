// topk.cu — wc_topk: compute/ranking.rs:15-80 (top_k, what vector_topk
// returns) on the device: the k live rows with the largest (or smallest)
// values in SQL order — NaN above every number, −0 equal to +0 — ties to
// the smaller dense id.  Each live value becomes an order-preserving
// 64-bit key; the live rows are compacted and sorted by key (CUB's radix
// sort, stable, so equal keys keep ascending ids) and the first k kept.
#include <cub/cub.cuh>

#include "operand.h"
#include "semiring.cuh"

namespace wc {

// The key of a value: larger key = ranked first.
__device__ inline uint64_t sql_key(double v, bool descending) {
  uint64_t k;
  if (v != v) {
    k = ~0ull;  // NaN: above every number
  } else {
    if (v == 0.0) v = 0.0;  // −0 and +0 are equal
    const uint64_t b = (uint64_t)__double_as_longlong(v);
    k = (b >> 63) ? ~b : (b | (1ull << 63));
  }
  return descending ? k : ~k;
}

template <class E> __device__ inline double as_f64(E v) { return (double)v; }

template <class E>
__global__ void topk_keys_kernel(const E* x, const uint64_t* tomb, uint32_t n, bool descending,
                                 uint64_t* keys, uint32_t* ids, uint8_t* live) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = sql_key(as_f64(x[i]), descending);
    ids[i] = i;
    live[i] = !(tomb && ((tomb[i >> 6] >> (i & 63)) & 1));
  }
}

template <class E>
static wc_status topk_typed(Ctx& ctx, const void* x, const uint64_t* tomb, uint64_t k, bool desc,
                            uint64_t* nodes_out, double* values_out, uint64_t* count) {
  const uint32_t n = (uint32_t)ctx.v->n;
  DevBuf *keys, *ids, *live, *k2, *i2, *num, *temp;
  WC_TRY(ctx.scratch(POOL_BATCH_0, (uint64_t)n * 8, &keys));
  WC_TRY(ctx.scratch(POOL_BATCH_1, (uint64_t)n * 4, &ids));
  WC_TRY(ctx.scratch(POOL_BATCH_2, n, &live));
  WC_TRY(ctx.scratch(POOL_BATCH_3, (uint64_t)n * 8, &k2));
  WC_TRY(ctx.scratch(POOL_BATCH_4, (uint64_t)n * 4 * 2, &i2));
  WC_TRY(ctx.scratch(POOL_TOPK_0, 16, &num));
  note_launch(), topk_keys_kernel<E><<<max_blocks(4), 256, 0, ctx.stream>>>(
      static_cast<const E*>(x), tomb, n, desc, keys->as<uint64_t>(), ids->as<uint32_t>(),
      live->as<uint8_t>());
  // Compact the live rows (keys and ids), then sort by key, descending.
  size_t t1 = 0, t2 = 0, t3 = 0;
  cub::DeviceSelect::Flagged(nullptr, t1, keys->as<uint64_t>(), live->as<uint8_t>(),
                             k2->as<uint64_t>(), num->as<int>(), (int)n, ctx.stream);
  cub::DeviceRadixSort::SortPairsDescending(nullptr, t3, keys->as<uint64_t>(), k2->as<uint64_t>(),
                                            ids->as<uint32_t>(), i2->as<uint32_t>(), (int)n, 0, 64,
                                            ctx.stream);
  t2 = std::max(t1, t3);
  WC_TRY(ctx.scratch(POOL_TOPK_1, t2 + 256, &temp));
  cub::DeviceSelect::Flagged(temp->ptr, t1, keys->as<uint64_t>(), live->as<uint8_t>(),
                             k2->as<uint64_t>(), num->as<int>(), (int)n, ctx.stream);
  cub::DeviceSelect::Flagged(temp->ptr, t1, ids->as<uint32_t>(), live->as<uint8_t>(),
                             i2->as<uint32_t>() + n, num->as<int>() + 1, (int)n, ctx.stream);
  int lives[2] = {0, 0};
  WC_CUDA(cudaMemcpyAsync(lives, num->ptr, 8, cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
  WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
  const int L = lives[0];
  // Sort the compacted (k2, i2+n) into (keys, ids).
  cub::DeviceRadixSort::SortPairsDescending(temp->ptr, t3, k2->as<uint64_t>(), keys->as<uint64_t>(),
                                            i2->as<uint32_t>() + n, ids->as<uint32_t>(), L, 0, 64,
                                            ctx.stream);
  const uint64_t kept = std::min<uint64_t>(k, (uint64_t)L);
  std::vector<uint32_t> top(kept);
  if (kept)
    WC_CUDA(cudaMemcpyAsync(top.data(), ids->ptr, kept * 4, cudaMemcpyDeviceToHost, ctx.stream),
            ctx.detail);
  WC_CUDA(cudaStreamSynchronize(ctx.stream), ctx.detail);
  for (uint64_t q = 0; q < kept; q++) {
    E val;
    WC_CUDA(cudaMemcpy(&val, static_cast<const E*>(x) + top[q], sizeof(E), cudaMemcpyDefault),
            ctx.detail);
    if (nodes_out) nodes_out[q] = top[q];
    if (values_out) values_out[q] = (double)val;
  }
  *count = kept;
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_topk(wc_version* v, const wc_call* call, wc_dtype dtype, const void* x,
                  const uint64_t* tombstones, uint64_t k, int32_t descending, uint64_t* nodes_out,
                  double* values_out, uint64_t* count) {
  if (!v || !x || !count) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  Operand X(POOL_X), T(POOL_MASK);
  WC_TRY(X.in(ctx, x, v->n * dtype_size(dtype)));
  const uint64_t* td = nullptr;
  if (tombstones) {
    WC_TRY(T.in(ctx, tombstones, ((v->n + 63) / 64) * 8));
    td = static_cast<const uint64_t*>(T.dev);
  }
  switch (dtype) {
    case WC_F64: WC_TRY(topk_typed<double>(ctx, X.dev, td, k, descending, nodes_out, values_out, count)); break;
    case WC_F32: WC_TRY(topk_typed<float>(ctx, X.dev, td, k, descending, nodes_out, values_out, count)); break;
    case WC_I64: WC_TRY(topk_typed<int64_t>(ctx, X.dev, td, k, descending, nodes_out, values_out, count)); break;
    case WC_BOOL: WC_TRY(topk_typed<uint8_t>(ctx, X.dev, td, k, descending, nodes_out, values_out, count)); break;
    default: return WC_DTYPE_MISMATCH;
  }
  return ctx.finish();
}

}  // extern "C"
