// Titarenko ring removal (remove_stripe_ti, src/tomocupy/processing/
// remove_stripe.py:296-307) on sinograms sino[z][p][x] (nz slices, nproj
// angles, n columns, in place):
//   v[z]  = mean over angles of sino[z] (a row of n), minus its column 0
//   v[z]  = irfft(rfft(v[z]) * rfft(gamma)),  gamma[k] = beta * q^|k|
//           (k the signed FFT frequency index, q = (1 - beta)/(1 + beta)),
//           gamma[0] -= 1
//   sino[z][p][x] += v[z][x] for x in the mask's column range.
// The column means reduce over angles with one thread per (slice, column)
// (coalesced along x, double accumulation in a fixed order, rounded to
// float32); the convolution follows the reference's types: a float32 real
// FFT of the float32 row (cuFFT R2C, as cupy.fft.rfft of a float32 array),
// promoted to complex128 and multiplied by the float64 gamma spectrum (1/n
// folded in, resident), then a float64 inverse (cuFFT Z2D); the add is one
// pass over the chunk, in double and rounded once to float32 like the
// reference's float32 + float64 in-place add.
#include <cmath>
#include <vector>

#include "common.cuh"

struct tcb_stripe_ti {
  size_t nproj, nz, n;
  long long m0, m1;  // masked column range [m0, m1)
  cufftHandle fwd = 0, inv = 0;
  float *v32 = nullptr;         // [nz, n] float32 rows (mean minus column 0)
  cufftComplex *V32 = nullptr;  // [nz, n/2+1] their float32 spectra
  double *v = nullptr;          // [nz, n]
  double2 *V = nullptr;         // [nz, n/2+1]
  double2 *G = nullptr;         // [n/2+1] rfft(gamma) / n
};

namespace tcb {
namespace {

// mean over angles minus the row's first mean: v[z][x] = float32(mean) - float32(mean_0)
__global__ void ti_colmean(float *__restrict__ v, const float *__restrict__ sino, int nproj,
                           int n, size_t zstride, size_t pstride) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  if (x >= n) return;
  const float *s = sino + (size_t)z * zstride + x;
  double acc = 0.0;
  for (int p = 0; p < nproj; p++) acc += (double)__ldg(s + (size_t)p * pstride);
  v[(size_t)z * n + x] = (float)(acc / nproj);
}

__global__ void ti_sub_first(float *__restrict__ v, int n) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  // column 0 is only read here (ti_zero_first clears it afterwards)
  if (x >= n) return;
  const float v0 = v[(size_t)z * n];
  if (x > 0) v[(size_t)z * n + x] = v[(size_t)z * n + x] - v0;
}

__global__ void ti_zero_first(float *__restrict__ v, int n) {
  v[(size_t)blockIdx.x * n] = 0.f;
}

// complex64 spectrum promoted to complex128, times the float64 gamma spectrum
__global__ void ti_mul(double2 *__restrict__ V, const cufftComplex *__restrict__ V32,
                       const double2 *__restrict__ G, int nc, size_t total) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const double ax = V32[t].x, ay = V32[t].y;
  const double2 g = G[t % nc];
  V[t] = make_double2(ax * g.x - ay * g.y, ax * g.y + ay * g.x);
}

__global__ void ti_add(float *__restrict__ sino, const double *__restrict__ v, int nproj, int n,
                       size_t zstride, size_t pstride, int m0, int m1) {
  const int x = m0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int p = blockIdx.y;
  const int z = blockIdx.z;
  if (x >= m1) return;
  float *s = sino + (size_t)z * zstride + (size_t)p * pstride + x;
  *s = (float)((double)*s + v[(size_t)z * n + x]);
}

void ti_release(tcb_stripe_ti *h) {
  if (h->fwd) cufftDestroy(h->fwd);
  if (h->inv) cufftDestroy(h->inv);
  cudaFree(h->v);
  cudaFree(h->V);
  cudaFree(h->G);
  cudaFree(h->v32);
  cudaFree(h->V32);
  h->v32 = nullptr;
  h->V32 = nullptr;
  h->fwd = h->inv = 0;
  h->v = nullptr;
  h->V = h->G = nullptr;
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_stripe_ti_mask(size_t n, double mask_size, long long *m0, long long *m1) {
  TCB_CHECK_ARG(m0 && m1, "tcb_stripe_ti_mask: null output");
  TCB_CHECK_ARG(n >= 1 && std::isfinite(mask_size), "tcb_stripe_ti_mask: bad arguments");
  // mask[:, n//2 - ms//2 : n//2 + ms//2] with ms = mask_size * n, Python slice rules
  const double ms = mask_size * (double)n;
  const double half = std::floor(ms / 2.0);
  long long a = (long long)((double)(n / 2) - half), b = (long long)((double)(n / 2) + half);
  const long long N = (long long)n;
  if (a < 0) a = std::max(0LL, a + N);
  if (b < 0) b = std::max(0LL, b + N);
  a = std::min(a, N);
  b = std::min(b, N);
  *m0 = a;
  *m1 = std::max(a, b);
  return TCB_OK;
}

extern "C" int tcb_stripe_ti_create(tcb_stripe_ti **out, size_t nproj, size_t nz, size_t n,
                                    double beta, double mask_size) {
  TCB_CHECK_ARG(out, "tcb_stripe_ti_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 1 && nz >= 1 && nz <= 65535 && n >= 2 && n < (1u << 30),
                "tcb_stripe_ti_create: bad sizes nproj=%zu nz=%zu n=%zu", nproj, nz, n);
  TCB_CHECK_ARG(beta > -1.0 && std::isfinite(beta), "tcb_stripe_ti_create: bad beta %g", beta);
  // the reference's irfft(rfft(v) * rfft(gamma)) returns n - 1 samples for
  // odd n, and its add then fails to broadcast
  TCB_CHECK_ARG(n % 2 == 0, "tcb_stripe_ti_create: n=%zu must be even", n);
  long long m0 = 0, m1 = 0;
  int st = tcb_stripe_ti_mask(n, mask_size, &m0, &m1);
  if (st != TCB_OK) return st;
  const size_t nc = n / 2 + 1;
  // gamma[k] = beta * ((1-beta)/(1+beta)) ** |fftfreq(n)[k] * n|, gamma[0] -= 1
  // (float64), and its real DFT by direct summation in long double
  const double q = (1.0 - beta) / (1.0 + beta);
  std::vector<double> gamma(n);
  for (size_t k = 0; k < n; k++) {
    const double f = (k < (n + 1) / 2) ? (double)k : (double)k - (double)n;  // fftfreq * n
    gamma[k] = beta * std::pow(q, std::fabs(f));
  }
  gamma[0] -= 1.0;
  std::vector<double2> G(nc);
  for (size_t j = 0; j < nc; j++) {
    long double re = 0, im = 0;
    for (size_t k = 0; k < n; k++) {
      const long double a = -2.0L * 3.14159265358979323846264338327950288L *
                            (long double)((j * k) % n) / (long double)n;
      re += gamma[k] * cosl(a);
      im += gamma[k] * sinl(a);
    }
    G[j] = make_double2((double)(re / n), (double)(im / n));
  }
  tcb_stripe_ti *h = new tcb_stripe_ti();
  h->nproj = nproj;
  h->nz = nz;
  h->n = n;
  h->m0 = m0;
  h->m1 = m1;
  auto fail = [&](int code) {
    ti_release(h);
    delete h;
    return code;
  };
  if (cudaMalloc(&h->v32, nz * n * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->V32, nz * nc * sizeof(cufftComplex)) != cudaSuccess ||
      cudaMalloc(&h->v, nz * n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->V, nz * nc * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&h->G, nc * sizeof(double2)) != cudaSuccess) {
    cudaGetLastError();
    set_error("tcb_stripe_ti_create: out of device memory");
    return fail(TCB_ERR_OUT_OF_MEMORY);
  }
  if (cudaMemcpy(h->G, G.data(), nc * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("tcb_stripe_ti_create: cudaMemcpy failed");
    return fail(TCB_ERR_CUDA);
  }
  int len[1] = {(int)n};
  cufftResult r = cufftPlanMany(&h->fwd, 1, len, nullptr, 1, (int)n, nullptr, 1, (int)nc,
                                CUFFT_R2C, (int)nz);
  if (r == CUFFT_SUCCESS)
    r = cufftPlanMany(&h->inv, 1, len, nullptr, 1, (int)nc, nullptr, 1, (int)n, CUFFT_Z2D,
                      (int)nz);
  if (r != CUFFT_SUCCESS) {
    set_error("tcb_stripe_ti_create: cufftPlanMany failed: %d", (int)r);
    return fail(r == CUFFT_ALLOC_FAILED ? TCB_ERR_OUT_OF_MEMORY : TCB_ERR_CUFFT);
  }
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_stripe_ti_apply_sino(tcb_stripe_ti *h, float *sino, size_t zstride,
                                        size_t pstride, void *stream) {
  TCB_CHECK_ARG(h, "tcb_stripe_ti_apply_sino: null handle");
  TCB_CHECK_ARG(h->v, "tcb_stripe_ti_apply_sino: handle was freed");
  TCB_CHECK_ARG(sino, "tcb_stripe_ti_apply_sino: null sino");
  // rows (z, p) must not overlap: slice-major or angle-major layouts
  TCB_CHECK_ARG(pstride >= h->n && zstride >= h->n &&
                    (zstride >= (h->nproj - 1) * pstride + h->n ||
                     pstride >= (h->nz - 1) * zstride + h->n),
                "tcb_stripe_ti_apply_sino: strides make rows overlap");
  TCB_CHECK_ARG(h->nproj <= 65535, "tcb_stripe_ti_apply_sino: nproj > 65535");
  cudaStream_t s = (cudaStream_t)stream;
  const int n = (int)h->n, nz = (int)h->nz, np = (int)h->nproj;
  const size_t nc = h->n / 2 + 1;
  StageTimer t("stripe_ti", s);
  ti_colmean<<<dim3(ceil_div(h->n, 256), nz), 256, 0, s>>>(h->v32, sino, np, n, zstride,
                                                             pstride);
  TCB_LAUNCH_CHECK();
  ti_sub_first<<<dim3(ceil_div(h->n, 256), nz), 256, 0, s>>>(h->v32, n);
  TCB_LAUNCH_CHECK();
  ti_zero_first<<<nz, 1, 0, s>>>(h->v32, n);
  TCB_LAUNCH_CHECK();
  TCB_CUFFT(cufftSetStream(h->fwd, s));
  TCB_CUFFT(cufftSetStream(h->inv, s));
  TCB_CUFFT(cufftExecR2C(h->fwd, h->v32, h->V32));
  ti_mul<<<ceil_div(h->nz * nc, 256), 256, 0, s>>>(h->V, h->V32, h->G, (int)nc, h->nz * nc);
  TCB_LAUNCH_CHECK();
  TCB_CUFFT(cufftExecZ2D(h->inv, (cufftDoubleComplex *)h->V, h->v));
  if (h->m1 > h->m0) {
    ti_add<<<dim3(ceil_div((size_t)(h->m1 - h->m0), 256), np, nz), 256, 0, s>>>(
        sino, h->v, np, n, zstride, pstride, (int)h->m0, (int)h->m1);
    TCB_LAUNCH_CHECK();
  }
  count_launch(h->m1 > h->m0 ? 5 : 4);
  return TCB_OK;
}

extern "C" int tcb_stripe_ti_destroy(tcb_stripe_ti *h) {
  if (!h) return TCB_OK;
  ti_release(h);
  delete h;
  return TCB_OK;
}
