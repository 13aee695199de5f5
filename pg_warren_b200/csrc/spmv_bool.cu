// spmv_bool.cu — the product kernels over bool vectors.
#include "spmv_impl.cuh"

namespace wc {
wc_status launch_pull_bool(const PullLaunch& L, const void* x, void* y) {
  return launch_typed<bool8>(L, x, y);
}
}  // namespace wc
