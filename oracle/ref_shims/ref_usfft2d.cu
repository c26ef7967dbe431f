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

// The reference's own take_x kernel (kernels_usfft2d.cu:5-18), launched with
// the operator's launch shape (cfunc_usfft2d.cu:37-40) into the caller's
// x, y [ntheta, deth, detw].
extern "C" void ref_take_x(size_t x, size_t y, size_t theta, float phi, int k, int deth0,
                           int detw, int deth, int ntheta, size_t stream) {
  dim3 BS2d(16, 8, 8);
  dim3 GS2d2(ceil(detw / (float)BS2d.x), ceil(deth / (float)BS2d.y),
             ceil(ntheta / (float)BS2d.z));
  take_x<<<GS2d2, BS2d, 0, (cudaStream_t)stream>>>((float *)x, (float *)y, (float *)theta, phi,
                                                   k, deth0, detw, deth, ntheta);
}
