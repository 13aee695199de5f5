// columns.cuh — per-column reductions over a grid, in a fixed order, for
// the kernels that run P columns at once (batched PageRank, the adjoint).
#pragma once

#include "runtime.cuh"

namespace wc {

// Per-column sums over the grid in a fixed order: lanes of one column
// (lane l holds column l mod P), warps, then blocks, by the last block to
// arrive.  Returns true in every thread of that block; its threads c < P
// then hold column c's totals.
template <int P>
__device__ inline bool reduce_columns(double& a, double& b, double* partials, unsigned* counter) {
  __shared__ double sa[8][P], sb[8][P];
  __shared__ bool last;
  const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (unsigned o = P; o < 32; o <<= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if (lane < P) {
    sa[wid][lane] = a;
    sb[wid][lane] = b;
  }
  __syncthreads();
  if (threadIdx.x < P) {
    double ta = 0.0, tb = 0.0;
    for (unsigned w = 0; w < blockDim.x / 32; w++) {
      ta += sa[w][threadIdx.x];
      tb += sb[w][threadIdx.x];
    }
    partials[((size_t)blockIdx.x * P + threadIdx.x) * 2] = ta;
    partials[((size_t)blockIdx.x * P + threadIdx.x) * 2 + 1] = tb;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  if (threadIdx.x < P) {
    double ta = 0.0, tb = 0.0;
    for (unsigned k = 0; k < gridDim.x; k++) {
      ta += __ldcg(partials + ((size_t)k * P + threadIdx.x) * 2);
      tb += __ldcg(partials + ((size_t)k * P + threadIdx.x) * 2 + 1);
    }
    a = ta;
    b = tb;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0;
  return true;
}

}  // namespace wc
