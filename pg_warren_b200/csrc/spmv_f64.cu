// spmv_f64.cu — the product kernels over f64 vectors.
#include "spmv_impl.cuh"

namespace wc {
wc_status launch_pull_f64(const PullLaunch& L, const void* x, void* y) {
  return launch_typed<double>(L, x, y);
}
}  // namespace wc
