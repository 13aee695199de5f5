// spmv_impl.cuh — kernels and dispatch of the product y = A ⊗ x (SpMV) and
// Y = A ⊗ X (SpMM), instantiated once per element type in spmv_<dtype>.cu.
#pragma once

#include "pull.cuh"
#include "pull_multi.cuh"
#include "product.h"

namespace wc {

template <class E, int S, class W>
__global__ void __launch_bounds__(kPullThreads, 3)
    spmv_pull_kernel(CsrView<W> A, const E* __restrict__ x, WriteEpi<E, S> epi, DeviceError* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  PullRing<E, W>* ring = reinterpret_cast<PullRing<E, W>*>(smem) + (threadIdx.x >> 5);
  pull_units<E, S, W>(A, x, epi, err, ring);
}

// SpMM, width > 1: the multi-column pull (pull_multi.cuh) over a block of
// P columns at a time — the row-split schedule, each column folded over
// the row's entries in ascending order (the reference's `fold`,
// compute/product/kernel.rs:184-198), long rows split into pieces combined
// in order — and the write (kernel.rs:200-240) per (row, column).
template <class E, int S> struct SpmmEpi {
  WriteArgs w;
  E* y;
  uint32_t width, c0;
  DeviceError* err;
  __device__ void cell(uint32_t row, uint32_t c, bool present, E t) {
    const uint32_t col = c0 + c;
    if (col >= width) return;
    E* out = y + (size_t)row * width + col;
    const E identity = Identity<E>::of(semiring_add(S));
    if (!mask_selects(w, row)) {
      if (w.replace) *out = identity;
      return;
    }
    if (w.accumulate < 0) {
      *out = present ? t : identity;
    } else if (present) {
      E r;
      int32_t s = apply_rt<E>(w.accumulate, *out, t, &r);
      if (s) raise(err, s, row);
      else *out = r;
    }
  }
};

template <class E, int S, class W, int P>
__global__ void __launch_bounds__(256)
    spmm_multi_kernel(CsrView<W> A, const E* __restrict__ x, E* y, uint32_t width, uint32_t c0,
                      WriteArgs w, DeviceError* err, Partial<E, semiring_add(S)>* carry) {
  SpmmEpi<E, S> epi{w, y, width, c0, err};
  pull_multi<E, S, W, P>(A, x + c0, epi, err, carry, width, min(P, width - c0));
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
    uint32_t blocks = (L.unit_count + 7) / 8;
    blocks = blocks < 1 ? 1 : (blocks > L.max_blocks ? L.max_blocks : blocks);
    auto* carry = static_cast<Partial<E, semiring_add(S)>*>(L.carry_multi);
    // Blocks of P columns: P the smallest power of two covering the width,
    // at most 32.
    for (uint32_t c0 = 0; c0 < L.width; c0 += 32) {
      const uint32_t cols = L.width - c0;
      if (cols >= 32)
        note_launch(), spmm_multi_kernel<E, S, W, 32><<<blocks, 256, 0, L.stream>>>(
            A, static_cast<const E*>(x), static_cast<E*>(y), L.width, c0, L.write, L.err, carry);
      else if (cols > 8)
        note_launch(), spmm_multi_kernel<E, S, W, 16><<<blocks, 256, 0, L.stream>>>(
            A, static_cast<const E*>(x), static_cast<E*>(y), L.width, c0, L.write, L.err, carry);
      else if (cols > 4)
        note_launch(), spmm_multi_kernel<E, S, W, 8><<<blocks, 256, 0, L.stream>>>(
            A, static_cast<const E*>(x), static_cast<E*>(y), L.width, c0, L.write, L.err, carry);
      else if (cols > 2)
        note_launch(), spmm_multi_kernel<E, S, W, 4><<<blocks, 256, 0, L.stream>>>(
            A, static_cast<const E*>(x), static_cast<E*>(y), L.width, c0, L.write, L.err, carry);
      else
        note_launch(), spmm_multi_kernel<E, S, W, 2><<<blocks, 256, 0, L.stream>>>(
            A, static_cast<const E*>(x), static_cast<E*>(y), L.width, c0, L.write, L.err, carry);
    }
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
