// pending.cu — entry points whose kernels are not built yet: they answer
// WC_UNSUPPORTED, the seam's "not served here" (the adapter keeps its
// native kernel).
#include "runtime.cuh"

extern "C" {

wc_status wc_pagerank_adjoint(wc_version*, const wc_call*, const wc_pagerank_opts*,
                              const uint64_t*, const uint64_t*, uint32_t, double, double*, double*,
                              uint32_t*) {
  return WC_UNSUPPORTED;
}
wc_status wc_topk(wc_version*, const wc_call*, wc_dtype, const void*, const uint64_t*, uint64_t,
                  int32_t, uint64_t*, double*, uint64_t*) {
  return WC_UNSUPPORTED;
}

}  // extern "C"
