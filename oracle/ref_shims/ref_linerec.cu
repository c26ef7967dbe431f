// Test-only shim around the reference's cfunc_linerec
// (src/include/cfunc_linerec.cuh:9-23, src/cuda/cfunc_linerec.cu:4-54).
#include "cfunc_linerec.cu"

extern "C" {
void *ref_create(size_t nproj, size_t nz, size_t n, size_t ncproj, size_t ncz) {
  return new cfunc_linerec(nproj, nz, n, ncproj, ncz);
}
void ref_backprojection(void *h, size_t f, size_t g, size_t theta, float phi,
                        int sz, size_t stream) {
  static_cast<cfunc_linerec *>(h)->backprojection(f, g, theta, phi, sz, stream);
}
void ref_backprojection_try(void *h, size_t f, size_t g, size_t theta, size_t sh,
                            float phi, int sz, size_t stream) {
  static_cast<cfunc_linerec *>(h)->backprojection_try(f, g, theta, sh, phi, sz,
                                                      stream);
}
void ref_backprojection_try_lamino(void *h, size_t f, size_t g, size_t theta,
                                   size_t phi, int sz, size_t stream) {
  static_cast<cfunc_linerec *>(h)->backprojection_try_lamino(f, g, theta, phi, sz,
                                                             stream);
}
void ref_destroy(void *h) { delete static_cast<cfunc_linerec *>(h); }
int ref_last_error(void) { return (int)cudaGetLastError(); }
}
