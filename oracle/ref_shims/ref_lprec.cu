// Test-only shim around the reference's cfunc_lprec
// (src/include/cfunc_lprec.cuh:9-49, src/cuda/cfunc_lprec.cu:14-160).
#include "cfunc_lprec.cu"

extern "C" {
void *ref_create(int nproj, int nz, int n, int ntheta, int nrho) {
  return new cfunc_lprec(nproj, nz, n, ntheta, nrho);
}
void ref_setgrids(void *h, size_t fz, size_t lp2p1, size_t lp2p2, size_t lp2p1w,
                  size_t lp2p2w, size_t C2lp1, size_t C2lp2, size_t lpids,
                  size_t wids, size_t cids, size_t nlpids, size_t nwids,
                  size_t ncids) {
  static_cast<cfunc_lprec *>(h)->setgrids(fz, lp2p1, lp2p2, lp2p1w, lp2p2w, C2lp1,
                                          C2lp2, lpids, wids, cids, nlpids, nwids,
                                          ncids);
}
void ref_backprojection(void *h, size_t f, size_t g, size_t stream) {
  static_cast<cfunc_lprec *>(h)->backprojection(f, g, stream);
}
void ref_destroy(void *h) { delete static_cast<cfunc_lprec *>(h); }
int ref_last_error(void) { return (int)cudaGetLastError(); }
}
