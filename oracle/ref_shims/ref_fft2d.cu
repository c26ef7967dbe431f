// Test-only shim around the reference's cfunc_fft2d
// (src/include/cfunc_fft2d.cuh:7-26, src/cuda/cfunc_fft2d.cu:4-63).
#include "cfunc_fft2d.cu"

extern "C" {
void *ref_create(size_t ntheta, size_t detw, size_t deth) {
  return new cfunc_fft2d(ntheta, detw, deth);
}
void ref_fwd(void *h, size_t g, size_t f, size_t stream) {
  static_cast<cfunc_fft2d *>(h)->fwd(g, f, stream);
}
void ref_destroy(void *h) { delete static_cast<cfunc_fft2d *>(h); }
int ref_last_error(void) { return (int)cudaGetLastError(); }
}
