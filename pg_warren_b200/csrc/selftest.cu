// selftest.cu — wc_selftest_bounded_wait: the bounded device wait the
// bulk-copy rings use (bulk.cuh, mbar_wait), made to run out on purpose on
// a barrier that no thread and no copy completes, so that a test can see the
// wait end with WC_DEVICE_TIMEOUT and the device stay usable.  Nothing is
// copied and nothing else waits, so the kernel ends as soon as its wait has
// given up.
#include "bulk.cuh"
#include "runtime.cuh"
#include "semiring.cuh"

namespace wc {

__global__ void bounded_wait_kernel(uint64_t limit_ns, int32_t* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival expected; none is ever made
    const bool done = mbar_wait(&bar, 0, limit_ns);
    *status = done ? WC_OK : WC_DEVICE_TIMEOUT;
  }
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_selftest_bounded_wait(const wc_call* call, uint32_t limit_us) {
  wc_error_detail* detail = call ? call->detail : nullptr;
  if (limit_us == 0 || limit_us > 2000000) return WC_INVALID_ARGUMENT;
  cudaStream_t stream = call && call->stream ? (cudaStream_t)call->stream : nullptr;
  int32_t* status = nullptr;
  WC_CUDA(cudaMallocHost(&status, sizeof(int32_t)), detail);
  *status = -1;
  note_launch(), bounded_wait_kernel<<<1, 32, 0, stream>>>(limit_us * 1000ull, status);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  const int32_t got = *status;
  cudaFreeHost(status);
  if (e != cudaSuccess) return cuda_status(e, detail, "bounded wait kernel");
  if (got == WC_DEVICE_TIMEOUT)
    set_message(detail, "a device wait gave up after %u us", limit_us);
  return (wc_status)got;
}

}  // extern "C"
