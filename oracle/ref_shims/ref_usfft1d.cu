// Test-only shim around the reference's cfunc_usfft1d
// (src/include/cfunc_usfft1d.cuh:7-34, src/cuda/cfunc_usfft1d.cu:5-86).
#include "cfunc_usfft1d.cu"

extern "C" {
void *ref_create(size_t n0, size_t n1, size_t n2, size_t deth) {
  return new cfunc_usfft1d(n0, n1, n2, deth);
}
void ref_fwd(void *h, size_t g, size_t f, float phi, size_t stream) {
  static_cast<cfunc_usfft1d *>(h)->fwd(g, f, phi, stream);
}
void ref_adj(void *h, size_t f, size_t g, float phi, size_t stream) {
  static_cast<cfunc_usfft1d *>(h)->adj(f, g, phi, stream);
}
void ref_destroy(void *h) { delete static_cast<cfunc_usfft1d *>(h); }
int ref_last_error(void) { return (int)cudaGetLastError(); }
}
