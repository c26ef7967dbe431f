// Test-only shim around the reference's cfunc_filter
// (src/include/cfunc_filter.cuh:9-23, src/cuda/cfunc_filter.cu:4-61).
#include "cfunc_filter.cu"

extern "C" {
void *ref_create(size_t nproj, size_t nz, size_t n) {
  return new cfunc_filter(nproj, nz, n);
}
void ref_filter(void *h, size_t g, size_t w, size_t stream) {
  static_cast<cfunc_filter *>(h)->filter(g, w, stream);
}
void ref_destroy(void *h) { delete static_cast<cfunc_filter *>(h); }
int ref_last_error(void) { return (int)cudaGetLastError(); }
}
