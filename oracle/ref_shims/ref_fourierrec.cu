// Test-only shim: exposes the reference's own cfunc_fourierrec class (compiled
// from the reference sources at build time, never copied) behind a tiny C ABI
// so the test suite can run the reference CUDA build on the same inputs as the
// new kernels. Built with -DHALF for the fp16 variant.
//
// Wraps src/include/cfunc_fourierrec.cuh:10-36 and src/cuda/cfunc_fourierrec.cu:4-94.
#include "cfunc_fourierrec.cu"

extern "C" {
void *ref_create(size_t nproj, size_t nz, size_t n, size_t theta) {
  return new cfunc_fourierrec(nproj, nz, n, theta);
}
void ref_backprojection(void *h, size_t f, size_t g, size_t stream) {
  static_cast<cfunc_fourierrec *>(h)->backprojection(f, g, stream);
}
void ref_destroy(void *h) { delete static_cast<cfunc_fourierrec *>(h); }
int ref_last_error(void) { return (int)cudaGetLastError(); }
}

// The reference's own takexy kernel (kernels_fourierrec.cuh:23-36), launched
// with the constructor's launch shape (cfunc_fourierrec.cu:43-49) into the
// caller's x, y [nproj, n]: the sample positions the reference grids with.
extern "C" void ref_takexy(size_t x, size_t y, size_t theta, size_t n, size_t nproj,
                           size_t stream) {
  dim3 dimBlock(32, 32, 1);
  dim3 GS2d0(ceil(n / 32.0), ceil(nproj / 32.0));
  takexy<<<GS2d0, dimBlock, 0, (cudaStream_t)stream>>>((float *)x, (float *)y, (float *)theta,
                                                        (int)n, (int)nproj);
}
