// Test-only shim around the reference's cfunc_usfft2d
// (src/include/cfunc_usfft2d.cuh:7-33, src/cuda/cfunc_usfft2d.cu:5-89).
#include "cfunc_usfft2d.cu"

extern "C" {
void *ref_create(size_t n0, size_t n1, size_t n2, size_t ntheta, size_t detw,
                 size_t deth) {
  return new cfunc_usfft2d(n0, n1, n2, ntheta, detw, deth);
}
void ref_fwd(void *h, size_t g, size_t f, size_t theta, float phi, int k, int deth0,
             size_t stream) {
  static_cast<cfunc_usfft2d *>(h)->fwd(g, f, theta, phi, k, deth0, stream);
}
void ref_adj(void *h, size_t f, size_t g, size_t theta, float phi, int k, int deth0,
             size_t stream) {
  static_cast<cfunc_usfft2d *>(h)->adj(f, g, theta, phi, k, deth0, stream);
}
void ref_destroy(void *h) { delete static_cast<cfunc_usfft2d *>(h); }
int ref_last_error(void) { return (int)cudaGetLastError(); }
}
