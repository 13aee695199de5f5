// spmv_i64.cu — the product kernels over i64 vectors.
#include "spmv_impl.cuh"

namespace wc {
wc_status launch_pull_i64(const PullLaunch& L, const void* x, void* y) {
  return launch_typed<int64_t>(L, x, y);
}
}  // namespace wc
