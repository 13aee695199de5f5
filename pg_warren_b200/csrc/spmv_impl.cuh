// spmv_impl.cuh — kernels and dispatch of the product y = A ⊗ x (SpMV) and
// Y = A ⊗ X (SpMM), instantiated once per element type in spmv_<dtype>.cu.
#pragma once

#include "pull.cuh"
#include "product.h"

namespace wc {

template <class E, int S, class W>
__global__ void __launch_bounds__(kPullThreads, 3)
    spmv_pull_kernel(CsrView<W> A, const E* __restrict__ x, WriteEpi<E, S> epi, DeviceError* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  PullRing<E, W>* ring = reinterpret_cast<PullRing<E, W>*>(smem) + (threadIdx.x >> 5);
  pull_units<E, S, W>(A, x, epi, err, ring);
}

// SpMM, width > 1: a warp per row, each lane folding columns lane, lane+32,
// ... over the row's entries in ascending order (the reference's `fold`,
// compute/product/kernel.rs:184-198), the first entry setting each sum.
template <class E, int S, class W>
__global__ void __launch_bounds__(256)
    spmm_rows_kernel(CsrView<W> A, uint32_t n, uint32_t width, const E* __restrict__ x, E* y,
                     WriteArgs w, DeviceError* err) {
  constexpr int ADD = semiring_add(S);
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const E identity = Identity<E>::of(ADD);
  for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps) {
    const uint32_t lo = __ldg(A.off + row), hi = __ldg(A.off + row + 1);
    const bool selected = mask_selects(w, row);
    for (uint32_t k0 = 0; k0 < width; k0 += 32) {
      const uint32_t k = k0 + lane;
      if (k >= width) continue;
      E* out = y + (size_t)row * width + k;
      if (!selected) {
        if (w.replace) *out = identity;
        continue;
      }
      E sum{};
      bool present = false;
      for (uint32_t e = lo; e < hi; e++) {
        const uint32_t j = __ldg(A.tgt + e);
        E p;
        int32_t s = EntryOf<E, S, W>::get(A, e, x[(size_t)j * width + k], &p);
        if (s) raise(err, s, row);
        if (present) {
          s = Apply<E, ADD>::go(sum, p, &sum);
          if (s) raise(err, s, row);
        } else {
          sum = p;
          present = true;
        }
      }
      if (w.accumulate < 0) {
        *out = present ? sum : identity;
      } else if (present) {
        E r;
        int32_t s = apply_rt<E>(w.accumulate, *out, sum, &r);
        if (s) raise(err, s, row);
        else *out = r;
      }
    }
  }
}

template <class E, int S, class W>
wc_status launch_one(const PullLaunch& L, const void* x, void* y) {
  CsrView<W> A{L.off, L.tgt, static_cast<const W*>(L.weights), L.units, L.unit_count,
               L.counters, L.carry};
  if (L.width == 1) {
    WriteEpi<E, S> epi{L.write, static_cast<E*>(y), L.err};
    constexpr size_t smem = pull_smem_bytes<E, W>();
    static const cudaError_t attr = cudaFuncSetAttribute(
        spmv_pull_kernel<E, S, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return cuda_status(attr, L.detail, "product kernel attributes");
    uint32_t blocks = (L.unit_count + kPullWarps - 1) / kPullWarps;
    blocks = blocks < 1 ? 1 : (blocks > L.max_blocks ? L.max_blocks : blocks);
    note_launch(), spmv_pull_kernel<E, S, W><<<blocks, kPullThreads, smem, L.stream>>>(
        A, static_cast<const E*>(x), epi, L.err);
  } else {
    uint32_t blocks = (L.n + 7) / 8;
    blocks = blocks < 1 ? 1 : (blocks > L.max_blocks ? L.max_blocks : blocks);
    note_launch(), spmm_rows_kernel<E, S, W><<<blocks, 256, 0, L.stream>>>(
        A, L.n, L.width, static_cast<const E*>(x), static_cast<E*>(y), L.write, L.err);
  }
  return cuda_status(cudaGetLastError(), L.detail, "product kernel launch");
}

template <class E, class W>
wc_status launch_semiring(const PullLaunch& L, const void* x, void* y) {
  switch (L.semiring) {
    case WC_PLUS_TIMES: return launch_one<E, WC_PLUS_TIMES, W>(L, x, y);
    case WC_MIN_PLUS: return launch_one<E, WC_MIN_PLUS, W>(L, x, y);
    case WC_MAX_PLUS: return launch_one<E, WC_MAX_PLUS, W>(L, x, y);
    case WC_MAX_TIMES: return launch_one<E, WC_MAX_TIMES, W>(L, x, y);
    case WC_MIN_TIMES: return launch_one<E, WC_MIN_TIMES, W>(L, x, y);
    case WC_LOR_LAND: return launch_one<E, WC_LOR_LAND, W>(L, x, y);
    case WC_ANY_PAIR: return launch_one<E, WC_ANY_PAIR, W>(L, x, y);
    case WC_PLUS_PAIR: return launch_one<E, WC_PLUS_PAIR, W>(L, x, y);
    case WC_PLUS_FIRST: return launch_one<E, WC_PLUS_FIRST, W>(L, x, y);
    case WC_PLUS_SECOND: return launch_one<E, WC_PLUS_SECOND, W>(L, x, y);
    case WC_MIN_FIRST: return launch_one<E, WC_MIN_FIRST, W>(L, x, y);
    case WC_MIN_SECOND: return launch_one<E, WC_MIN_SECOND, W>(L, x, y);
    case WC_MAX_SECOND: return launch_one<E, WC_MAX_SECOND, W>(L, x, y);
  }
  return WC_UNKNOWN_SEMIRING;
}

template <class E>
wc_status launch_typed(const PullLaunch& L, const void* x, void* y) {
  switch (L.weight_kind) {
    case WEIGHTS_F64: return launch_semiring<E, double>(L, x, y);
    case WEIGHTS_I32: return launch_semiring<E, int32_t>(L, x, y);
    default: return launch_semiring<E, void>(L, x, y);
  }
}

}  // namespace wc
