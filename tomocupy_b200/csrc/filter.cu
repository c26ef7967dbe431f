// FBP filter operator: real rows of length n are transformed (R2C), each
// slice's spectrum is multiplied by its own complex weight w[z, :], and the
// rows are transformed back (C2R) in place.
//
// Same contract as cfunc_filter::filter (src/cuda/cfunc_filter.cu:49-61):
// the 1/n normalisation is folded into w by the caller
// (reconstruction/fbp_filter.py:87).  The FLOAT16 variant keeps the caller's
// buffers in fp16 but transforms in fp32.
#include <cuda_fp16.h>

#include "common.cuh"

struct tcb_filter {
  size_t nproj, nz, n;
  int precision;
  cufftHandle fwd = 0, inv = 0;
  float2 *ge = nullptr;   // [nz*nproj, n/2+1] spectrum scratch
  float *g32 = nullptr;   // fp32 staging of the rows (FLOAT16 only)
};

namespace tcb {
namespace {

__global__ void mulw_kernel(float2 *__restrict__ ge, const float2 *__restrict__ w,
                            int nc, int nproj, size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int k = (int)(i % nc);
  size_t row = i / nc;
  int z = (int)(row / nproj);
  float2 g = ge[i];
  float2 c = w[(size_t)z * nc + k];
  ge[i] = make_float2(g.x * c.x - g.y * c.y, g.x * c.y + g.y * c.x);
}

__global__ void mulw_half_kernel(float2 *__restrict__ ge, const __half2 *__restrict__ w,
                                 int nc, int nproj, size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int k = (int)(i % nc);
  size_t row = i / nc;
  int z = (int)(row / nproj);
  float2 g = ge[i];
  float2 c = __half22float2(w[(size_t)z * nc + k]);
  ge[i] = make_float2(g.x * c.x - g.y * c.y, g.x * c.y + g.y * c.x);
}

__global__ void half_to_float_kernel(float *__restrict__ dst, const __half *__restrict__ src,
                                     size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) dst[i] = __half2float(src[i]);
}

__global__ void float_to_half_kernel(__half *__restrict__ dst, const float *__restrict__ src,
                                     size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) dst[i] = __float2half_rn(src[i]);
}

void filter_release(tcb_filter *h) {
  if (h->fwd) cufftDestroy(h->fwd);
  if (h->inv) cufftDestroy(h->inv);
  if (h->ge) cudaFree(h->ge);
  if (h->g32) cudaFree(h->g32);
  h->fwd = h->inv = 0;
  h->ge = nullptr;
  h->g32 = nullptr;
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_filter_create(tcb_filter **out, size_t nproj, size_t nz, size_t n,
                                 int precision) {
  TCB_CHECK_ARG(out, "tcb_filter_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 1 && nz >= 1 && n >= 2 && n % 2 == 0,
                "tcb_filter_create: bad sizes nproj=%zu nz=%zu n=%zu (n must be even)",
                nproj, nz, n);
  TCB_CHECK_ARG(precision == TCB_FLOAT32 || precision == TCB_FLOAT16,
                "tcb_filter_create: bad precision %d", precision);
  TCB_CHECK_ARG(nproj * nz < (1ull << 31), "tcb_filter_create: batch too large");
  tcb_filter *h = new tcb_filter();
  h->nproj = nproj;
  h->nz = nz;
  h->n = n;
  h->precision = precision;
  int rank_n[1] = {(int)n};
  int batch = (int)(nproj * nz);
  int nc = (int)(n / 2 + 1);
  int st = TCB_OK;
  auto fail = [&](int code) {
    filter_release(h);
    delete h;
    return code;
  };
  cudaError_t e = cudaMalloc(&h->ge, (size_t)batch * nc * sizeof(float2));
  if (e != cudaSuccess) {
    set_error("tcb_filter_create: cudaMalloc(%zu) failed: %s",
              (size_t)batch * nc * sizeof(float2), cudaGetErrorString(e));
    return fail(TCB_ERR_OUT_OF_MEMORY);
  }
  if (precision == TCB_FLOAT16) {
    e = cudaMalloc(&h->g32, (size_t)batch * n * sizeof(float));
    if (e != cudaSuccess) {
      set_error("tcb_filter_create: cudaMalloc failed: %s", cudaGetErrorString(e));
      return fail(TCB_ERR_OUT_OF_MEMORY);
    }
  }
  cufftResult r = cufftPlanMany(&h->fwd, 1, rank_n, rank_n, 1, (int)n, &nc, 1, nc,
                                CUFFT_R2C, batch);
  if (r == CUFFT_SUCCESS)
    r = cufftPlanMany(&h->inv, 1, rank_n, &nc, 1, nc, rank_n, 1, (int)n, CUFFT_C2R, batch);
  if (r != CUFFT_SUCCESS) {
    set_error("tcb_filter_create: cufftPlanMany failed: %d", (int)r);
    return fail(r == CUFFT_ALLOC_FAILED ? TCB_ERR_OUT_OF_MEMORY : TCB_ERR_CUFFT);
  }
  (void)st;
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_filter_apply(tcb_filter *h, void *g, const void *w, void *stream) {
  TCB_CHECK_ARG(h, "tcb_filter_apply: null handle");
  TCB_CHECK_ARG(h->ge, "tcb_filter_apply: handle was freed");
  TCB_CHECK_ARG(g && w, "tcb_filter_apply: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  TCB_CUFFT(cufftSetStream(h->fwd, s));
  TCB_CUFFT(cufftSetStream(h->inv, s));
  size_t nc = h->n / 2 + 1;
  size_t total_c = h->nproj * h->nz * nc;
  size_t total_r = h->nproj * h->nz * h->n;
  float *rows = (float *)g;
  if (h->precision == TCB_FLOAT16) {
    half_to_float_kernel<<<ceil_div(total_r, 256), 256, 0, s>>>(h->g32, (const __half *)g,
                                                                 total_r);
    TCB_LAUNCH_CHECK();
    count_launch();
    rows = h->g32;
  }
  {
    StageTimer st("filter_r2c", s);
    TCB_CUFFT(cufftExecR2C(h->fwd, rows, (cufftComplex *)h->ge));
  }
  {
    StageTimer st("filter_mulw", s);
    if (h->precision == TCB_FLOAT16)
      mulw_half_kernel<<<ceil_div(total_c, 256), 256, 0, s>>>(h->ge, (const __half2 *)w,
                                                              (int)nc, (int)h->nproj, total_c);
    else
      mulw_kernel<<<ceil_div(total_c, 256), 256, 0, s>>>(h->ge, (const float2 *)w, (int)nc,
                                                         (int)h->nproj, total_c);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  {
    StageTimer st("filter_c2r", s);
    TCB_CUFFT(cufftExecC2R(h->inv, (cufftComplex *)h->ge, rows));
  }
  if (h->precision == TCB_FLOAT16) {
    float_to_half_kernel<<<ceil_div(total_r, 256), 256, 0, s>>>((__half *)g, h->g32,
                                                                 total_r);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

extern "C" int tcb_filter_destroy(tcb_filter *h) {
  if (!h) return TCB_OK;
  filter_release(h);
  delete h;
  return TCB_OK;
}
