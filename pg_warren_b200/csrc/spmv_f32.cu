// spmv_f32.cu — the product kernels over f32 vectors.
#include "spmv_impl.cuh"

namespace wc {
wc_status launch_pull_f32(const PullLaunch& L, const void* x, void* y) {
  return launch_typed<float>(L, x, y);
}
}  // namespace wc
