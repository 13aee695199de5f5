// vector.cu — wc_vector_reduce and wc_vector_norm_diff: compute/reduce.rs
// (vector_reduce, vector_norm_diff) on the device, to the bit.
//
// The reference reduces chunks of 65,536 elements (row-major) in parallel,
// each chunk's sum taken in element order from +0, then the chunks'
// results in chunk order (reduce.rs:20, 195-212, 250-268).  A float sum's
// value depends on that order, so each chunk's sum is one dependent chain
// here too: a block per chunk, its warps staging the chunk's terms in
// shared memory (2,048 at a time, double-buffered) while one thread adds
// them in order.  A row the tombstones skip contributes the term -0.0,
// which leaves every sum as it was (s + -0.0 = s for every s, NaN and +0
// included).  Max and min keep the first of equal elements in SQL order
// (NaN above every number), so they reduce in any order on (value, index).
#include <cmath>

#include "operand.h"
#include "runtime.cuh"
#include "semiring.cuh"

namespace wc {

constexpr uint32_t kReduceChunk = 1u << 16;  // reduce.rs:20
constexpr uint32_t kStage = 2048;
// The pointer of a vector with no elements (never read).
static const double kNoElements = 0.0;

// The i-th element of the operand (0 past `len`: a shorter vector of a
// norm difference is padded with zeros, reduce.rs:229-238).
struct Elems {
  const void* p;
  uint64_t len;
  int32_t dtype;
  __device__ double at(uint64_t i) const {
    if (i >= len) return 0.0;
    switch (dtype) {
      case WC_F64: return static_cast<const double*>(p)[i];
      case WC_F32: return (double)static_cast<const float*>(p)[i];
      case WC_I64: return (double)static_cast<const int64_t*>(p)[i];
      default: return static_cast<const uint8_t*>(p)[i] ? 1.0 : 0.0;
    }
  }
};

// What one element contributes: the term of a sum, or the element itself.
struct Term {
  Elems a, b;       // b.p NULL: a reduction of a alone
  uint32_t width;
  const uint64_t* tomb;
  int32_t op;       // wc_reduction
  __device__ bool kept(uint64_t i) const {
    if (!tomb) return true;
    const uint64_t row = i / width;
    return !((tomb[row >> 6] >> (row & 63)) & 1);
  }
  __device__ double value(uint64_t i) const {
    const double v = a.at(i);
    return b.p ? v - b.at(i) : v;
  }
};

__device__ inline bool sql_gt(double a, double b) { return sql_cmp_f(a, b) > 0; }

// The term element i adds to a sum (-0.0 past the chunk or for a skipped row).
__device__ inline double term_of(const Term& t, uint64_t i, uint64_t c1) {
  if (i >= c1 || !t.kept(i)) return -0.0;
  const double v = t.value(i);
  switch (t.op) {
    case WC_REDUCE_L1: return fabs(v);
    case WC_REDUCE_L2: return v * v;
    case WC_REDUCE_NNZ: return v != 0.0 ? 1.0 : 0.0;  // NaN is non-zero
    default: return v;
  }
}

// Sums of terms (sum, l1, l2, nnz): block c reduces chunk c into partial[c].
__global__ void __launch_bounds__(256) reduce_sum_kernel(Term t, uint64_t len, double* partial) {
  __shared__ double stage[2][kStage];
  const uint64_t c0 = (uint64_t)blockIdx.x * kReduceChunk;
  const uint64_t c1 = min(len, c0 + kReduceChunk);
  const uint32_t rounds = (uint32_t)((c1 - c0 + kStage - 1) / kStage);
  // Threads [first, blockDim) stage round r.
  auto fill = [&](uint32_t r, uint32_t first) {
    double* s = stage[r & 1];
    for (uint32_t q = threadIdx.x - first; q < kStage; q += blockDim.x - first)
      s[q] = term_of(t, c0 + (uint64_t)r * kStage + q, c1);
  };
  double sum = 0.0;
  fill(0, 0);
  __syncthreads();
  for (uint32_t r = 0; r < rounds; r++) {
    // Thread 0 adds round r in order while warps 1.. stage round r + 1.
    if (threadIdx.x == 0) {
      const double* s = stage[r & 1];
#pragma unroll 16
      for (uint32_t q = 0; q < kStage; q++) sum = sum + s[q];
    } else if (threadIdx.x >= 32 && r + 1 < rounds) {
      fill(r + 1, 32);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sum;
}

// Max / min (Linf: max of |difference|): the first of the SQL-greatest
// (least) elements of chunk c, as (value, present) in partial[2c .. 2c+1].
__global__ void __launch_bounds__(256) reduce_extreme_kernel(Term t, uint64_t len, bool greatest,
                                                             bool absolute, double* partial) {
  __shared__ double sv[256];
  __shared__ unsigned long long si[256];
  const uint64_t c0 = (uint64_t)blockIdx.x * kReduceChunk;
  const uint64_t c1 = min(len, c0 + kReduceChunk);
  const unsigned long long kNone = ~0ull;
  double best = 0.0;
  unsigned long long at = kNone;
  // better(v, i) over (best, at): strictly beyond in SQL order, or equal
  // and earlier.
  auto take = [&](double v, unsigned long long i) {
    if (at == kNone) {
      best = v, at = i;
      return;
    }
    const int c = sql_cmp_f(v, best);
    if ((greatest ? c > 0 : c < 0) || (c == 0 && i < at)) best = v, at = i;
  };
  for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
    if (!t.kept(i)) continue;
    const double v = t.value(i);
    take(absolute ? fabs(v) : v, i);
  }
  sv[threadIdx.x] = best;
  si[threadIdx.x] = at;
  __syncthreads();
  for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o && si[threadIdx.x + o] != kNone) {
      take(sv[threadIdx.x + o], si[threadIdx.x + o]);
      sv[threadIdx.x] = best;
      si[threadIdx.x] = at;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = best;
    partial[2 * blockIdx.x + 1] = at == kNone ? 0.0 : 1.0;
  }
}

// The chunks' results in chunk order (reduce.rs:262-268): one thread.
__global__ void reduce_combine_kernel(const double* partial, uint32_t chunks, int32_t op,
                                      double* out) {
  if (blockIdx.x || threadIdx.x) return;
  if (op == WC_REDUCE_MAX || op == WC_REDUCE_MIN) {
    double best = 0.0;
    bool any = false;
    for (uint32_t c = 0; c < chunks; c++) {
      if (partial[2 * c + 1] == 0.0) continue;
      const double v = partial[2 * c];
      if (!any) best = v, any = true;
      else if (op == WC_REDUCE_MAX ? sql_gt(v, best) : sql_cmp_f(v, best) < 0) best = v;
    }
    out[0] = best;
    out[1] = any ? 0.0 : 1.0;  // NULL: no element
    return;
  }
  double sum = 0.0;
  for (uint32_t c = 0; c < chunks; c++) sum = sum + partial[c];
  out[0] = op == WC_REDUCE_L2 ? sqrt(sum) : sum;
  out[1] = 0.0;
}

static uint32_t elem_size(int32_t dtype) {
  switch (dtype) {
    case WC_F64: case WC_I64: return 8;
    case WC_F32: return 4;
    case WC_BOOL: return 1;
    default: return 0;
  }
}

static wc_status run_reduce(Ctx& ctx, const Term& t, uint64_t len, int32_t op, double* result,
                            int32_t* is_null) {
  const uint32_t chunks = (uint32_t)std::max<uint64_t>(1, (len + kReduceChunk - 1) / kReduceChunk);
  DevBuf *pb, *ob;
  WC_TRY(ctx.scratch(POOL_VEC_PARTIAL, (uint64_t)chunks * 16, &pb));
  WC_TRY(ctx.scratch(POOL_VEC_RESULT, 16, &ob));
  double* partial = pb->as<double>();
  if (op == WC_REDUCE_MAX || op == WC_REDUCE_MIN)
    note_launch(), reduce_extreme_kernel<<<chunks, 256, 0, ctx.stream>>>(
        t, len, op == WC_REDUCE_MAX, t.b.p != nullptr, partial);
  else
    note_launch(), reduce_sum_kernel<<<chunks, 256, 0, ctx.stream>>>(t, len, partial);
  note_launch(), reduce_combine_kernel<<<1, 32, 0, ctx.stream>>>(partial, chunks, op, ob->as<double>());
  double host[2];
  WC_CUDA(cudaMemcpyAsync(host, ob->ptr, 16, cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
  WC_TRY(ctx.finish());
  *result = host[0];
  if (is_null) *is_null = host[1] != 0.0;
  return WC_OK;
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_vector_reduce(wc_version* v, const wc_call* call, wc_dtype dtype, const void* x,
                           uint32_t width, const uint64_t* tombstone_words, wc_reduction reduction,
                           double* result, int32_t* is_null) {
  if (!v || !result || width == 0 || (v->n && !x)) return WC_INVALID_ARGUMENT;
  if (reduction < WC_REDUCE_SUM || reduction > WC_REDUCE_NNZ) return WC_INVALID_ARGUMENT;
  const uint32_t size = elem_size(dtype);
  if (!size) return WC_DTYPE_MISMATCH;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  const uint64_t len = v->n * width;
  Operand X(POOL_X), T(POOL_MASK);
  const void* xd = &kNoElements;  // never read: no element lies below len = 0
  if (len) {
    WC_TRY(X.in(ctx, x, len * size));
    xd = X.dev;
  }
  const uint64_t* td = nullptr;
  if (tombstone_words && v->n) {
    WC_TRY(T.in(ctx, tombstone_words, ((v->n + 63) / 64) * 8));
    td = static_cast<const uint64_t*>(T.dev);
  }
  Term t{Elems{xd, len, dtype}, Elems{nullptr, 0, 0}, width, td, reduction};
  return run_reduce(ctx, t, len, reduction, result, is_null);
}

wc_status wc_vector_norm_diff(wc_version* v, const wc_call* call, wc_dtype dtype_a, const void* a,
                              uint64_t id_space_a, wc_dtype dtype_b, const void* b,
                              uint64_t id_space_b, uint32_t width, wc_norm norm, double* result) {
  if (!v || !result || width == 0 || (id_space_a && !a) || (id_space_b && !b))
    return WC_INVALID_ARGUMENT;
  if (norm < WC_NORM_L1 || norm > WC_NORM_LINF) return WC_INVALID_ARGUMENT;
  const uint32_t sa = elem_size(dtype_a), sb = elem_size(dtype_b);
  if (!sa || !sb) return WC_DTYPE_MISMATCH;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  const uint64_t la = id_space_a * width, lb = id_space_b * width;
  Operand A(POOL_X), B(POOL_Y);
  // A vector with no elements reads as zeros; its pointer is never read,
  // but b's marks the reduction as a difference.
  const void* ad = &kNoElements;
  const void* bd = &kNoElements;
  if (la) {
    WC_TRY(A.in(ctx, a, la * sa));
    ad = A.dev;
  }
  if (lb) {
    WC_TRY(B.in(ctx, b, lb * sb));
    bd = B.dev;
  }
  const int32_t op = norm == WC_NORM_L1 ? WC_REDUCE_L1 : norm == WC_NORM_L2 ? WC_REDUCE_L2
                                                                           : WC_REDUCE_MAX;
  Term t{Elems{ad, la, dtype_a}, Elems{bd, lb, dtype_b}, width, nullptr, op};
  int32_t null = 0;
  WC_TRY(run_reduce(ctx, t, std::max(la, lb), op, result, &null));
  if (null) *result = 0.0;  // reduce.rs:203: the norm of nothing is 0
  return WC_OK;
}

}  // extern "C"
