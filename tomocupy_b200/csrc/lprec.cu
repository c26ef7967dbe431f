// Log-polar (lprec) backprojector.
//
// Same algorithm as cfunc_lprec (src/cuda/cfunc_lprec.cu:103-160,
// src/include/kernels_lprec.cuh): cubic B-spline prefilter of the sinograms
// along the detector and then the angle axis, cubic interpolation from the
// polar to the log-polar grid of each of three angular spans (hardware
// linear texture fetches combined with B-spline weights, the published
// "fast third-order texture filtering" construction), a 2D R2C FFT
// convolution with the precomputed kernel fZ, and cubic interpolation from
// log-polar to Cartesian coordinates accumulated into the slices.
//
// B200 design:
//  * the prefilter needs no global transposes: the detector-axis recursion
//    runs on 32x32 shared-memory tiles per warp (one row per lane, state
//    carried across tiles), the angle-axis recursion runs one column per lane
//    with coalesced row loads;
//  * the 2/(nrho*ntheta) normalisation is folded into an internal copy of fZ
//    (one pass fewer per span);
//  * interpolation kernels use flat 1D grids over the point lists;
//  * for power-of-two nrho and ntheta in [256, 8192] the FFT convolution runs
//    on the library's own FFT: two log-polar slices packed as one complex
//    image (the kernel's Hermitian extension H maps each real slice to a real
//    result), rows forward, then per column forward, times H, inverse, then
//    rows inverse with the real and imaginary parts written back to the two
//    slices.  cuFFT's C2R takes the zero-frequency column of the product
//    through its Hermitian part, so H's column 0 is (fZ(k, 0) +
//    conj(fZ(-k, 0))) / 2.
// Texture objects and layered CUDA arrays are used exactly as the reference
// uses them, because its parity depends on the texture unit's 8-bit
// fixed-point filtering weights.
#include <cuda_fp16.h>

#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "fft_pow2.cuh"

struct tcb_lprec {
  int nproj, nz, n, ntheta, nrho, precision;
  // grids borrowed from the caller (setgrids), as in the reference
  const float2 *fz = nullptr;
  const float *lp2p1 = nullptr, *lp2p2 = nullptr, *lp2p1w = nullptr, *lp2p2w = nullptr;
  const float *C2lp1 = nullptr, *C2lp2 = nullptr;
  const int *lpids = nullptr, *wids = nullptr, *cids = nullptr;
  int nlpids = 0, nwids = 0, ncids = 0;
  // owned
  float2 *fzs = nullptr;  // fZ * 2/(nrho*ntheta)
  float *fl = nullptr;    // [nz, nrho, ntheta]
  float2 *flc = nullptr;  // [nz, nrho, ntheta/2+1]
  float *g32 = nullptr;   // fp32 staging (FLOAT16 only)
  float *f32 = nullptr;   // fp32 output staging (FLOAT16 only)
  cudaArray_t ga = nullptr, fla = nullptr;
  cudaTextureObject_t texg = 0, texfl = 0;
  cufftHandle fwd = 0, inv = 0;
  // own-FFT convolution
  bool own = false;
  float2 *t1 = nullptr;   // [pairs][ntheta/8][nrho][8] row spectra
  float2 *t2 = nullptr;   // [pairs][nrho][ntheta] filtered, rows not yet inverted
  float2 *h0 = nullptr;   // [nrho] Hermitian part of column 0 of fzs
  float2 *twr = nullptr, *twt = nullptr;  // twiddles of lengths nrho, ntheta
};

namespace tcb {
namespace lp {

constexpr float POLE = -0.267949192431123f;

// ---- cubic B-spline prefilter (kernels_lprec.cuh:65-110 arithmetic) ----
__device__ __forceinline__ float lambda_gain() {
  return (1.0f - POLE) * (1.0f - 1.0f / POLE);
}

// Recursion along contiguous rows: one warp, 32 rows, 32-column tiles.
__global__ void prefilter_rows(float *__restrict__ g, int len, long long nrows) {
  __shared__ float tile[8][32][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  long long row0 = ((long long)blockIdx.x * 8 + w) * 32;
  if (row0 >= nrows) return;
  float (*t)[33] = tile[w];
  const int nr = (int)min(32LL, nrows - row0);
  float *base = g + row0 * len;
  const float L = lambda_gain();
  const int horizon = 12 < len ? 12 : len;
  // causal pass
  float prev = 0.f;
  for (int c0 = 0; c0 < len; c0 += 32) {
    int nc = min(32, len - c0);
    for (int r = 0; r < nr; r++)
      if (lane < nc) t[r][lane] = base[(long long)r * len + c0 + lane];
    __syncwarp();
    if (lane < nr) {
      int k0 = 0;
      if (c0 == 0) {
        // InitialCausalCoefficient: Sum = c0 + sum_{k<H} Pole^{k+1} c_k
        float zn = POLE, sum = t[lane][0];
        const float *rowp = base + (long long)lane * len;
        for (int k = 0; k < horizon; k++) {
          float ck = (k < 32) ? t[lane][k] : rowp[k];
          sum += zn * ck;
          zn *= POLE;
        }
        prev = L * sum;
        t[lane][0] = prev;
        k0 = 1;
      }
      for (int k = k0; k < nc; k++) {
        prev = L * t[lane][k] + POLE * prev;
        t[lane][k] = prev;
      }
    }
    __syncwarp();
    for (int r = 0; r < nr; r++)
      if (lane < nc) base[(long long)r * len + c0 + lane] = t[r][lane];
    __syncwarp();
  }
  // anticausal pass (from the end)
  int last0 = ((len - 1) / 32) * 32;
  for (int c0 = last0; c0 >= 0; c0 -= 32) {
    int nc = min(32, len - c0);
    for (int r = 0; r < nr; r++)
      if (lane < nc) t[r][lane] = base[(long long)r * len + c0 + lane];
    __syncwarp();
    if (lane < nr) {
      int k1 = nc - 1;
      if (c0 == last0) {
        prev = (POLE / (POLE - 1.0f)) * t[lane][k1];
        t[lane][k1] = prev;
        k1--;
      }
      for (int k = k1; k >= 0; k--) {
        prev = POLE * (prev - t[lane][k]);
        t[lane][k] = prev;
      }
    }
    __syncwarp();
    for (int r = 0; r < nr; r++)
      if (lane < nc) base[(long long)r * len + c0 + lane] = t[r][lane];
    __syncwarp();
  }
}

// Recursion along columns (stride `width`) of [nz][len][width]: one column per
// thread, consecutive threads on consecutive columns (coalesced rows).
__global__ void prefilter_cols(float *__restrict__ g, int width, int len, int nz) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y;
  if (x >= width || z >= nz) return;
  float *c = g + (size_t)z * width * len + x;
  const float L = lambda_gain();
  const int horizon = 12 < len ? 12 : len;
  float zn = POLE, sum = c[0];
  for (int k = 0; k < horizon; k++) {
    sum += zn * c[(size_t)k * width];
    zn *= POLE;
  }
  float prev = L * sum;
  c[0] = prev;
  for (int k = 1; k < len; k++) {
    prev = L * c[(size_t)k * width] + POLE * prev;
    c[(size_t)k * width] = prev;
  }
  prev = (POLE / (POLE - 1.0f)) * c[(size_t)(len - 1) * width];
  c[(size_t)(len - 1) * width] = prev;
  for (int k = len - 2; k >= 0; k--) {
    prev = POLE * (prev - c[(size_t)k * width]);
    c[(size_t)k * width] = prev;
  }
}

// ---- cubic interpolation through linear texture fetches ----
__device__ __forceinline__ void bspline_w(float fr, float w[4]) {
  const float one_frac = 1.0f - fr;
  const float squared = fr * fr;
  const float one_sqd = one_frac * one_frac;
  w[0] = 1.0f / 6.0f * one_sqd * one_frac;
  w[1] = 2.0f / 3.0f - 0.5f * squared * (2.0f - fr);
  w[2] = 2.0f / 3.0f - 0.5f * one_sqd * (2.0f - one_frac);
  w[3] = 1.0f / 6.0f * squared * fr;
}

__device__ __forceinline__ float cubic_fetch(cudaTextureObject_t tex, float x, float y, int z,
                                             int n0, int n1) {
  const float ix = floor(x);
  const float fx = x - ix;
  float wx[4];
  bspline_w(fx, wx);
  const float g0x = wx[0] + wx[1];
  const float g1x = wx[2] + wx[3];
  const float h0x = ((wx[1] / g0x - 0.5f) + ix) / float(n0);
  const float h1x = ((wx[3] / g1x + 1.5f) + ix) / float(n0);
  const float iy = floor(y);
  const float fy = y - iy;
  float wy[4];
  bspline_w(fy, wy);
  const float g0y = wy[0] + wy[1];
  const float g1y = wy[2] + wy[3];
  const float h0y = ((wy[1] / g0y - 0.5f) + iy) / float(n1);
  const float h1y = ((wy[3] / g1y + 1.5f) + iy) / float(n1);
  float t00 = tex2DLayered<float>(tex, h0x, h0y, z);
  float t10 = tex2DLayered<float>(tex, h1x, h0y, z);
  float t01 = tex2DLayered<float>(tex, h0x, h1y, z);
  float t11 = tex2DLayered<float>(tex, h1x, h1y, z);
  t00 = g0y * t00 + g1y * t01;
  t10 = g0y * t10 + g1y * t11;
  return g0x * t00 + g1x * t10;
}

// f[z*step + ids[t]] += cubic(tex, x[t], y[t], layer z)
__global__ void interp_points(cudaTextureObject_t tex, float *__restrict__ f,
                              const float *__restrict__ x, const float *__restrict__ y, int np,
                              int n0, int n1, const int *__restrict__ ids, long long step) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y;
  if (t >= np) return;
  f[z * step + ids[t]] += cubic_fetch(tex, x[t], y[t], z, n0, n1);
}

// spectrum *= fzs (fZ pre-scaled by 2/(nrho*ntheta))
__global__ void mul_fz(float2 *__restrict__ flc, const float2 *__restrict__ fz, long long plane,
                       long long total) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  float2 y = flc[i], x = fz[i % plane];
  flc[i] = make_float2(y.x * x.x - y.y * x.y, y.x * x.y + y.y * x.x);
}

__global__ void scale_fz(float2 *__restrict__ dst, const float2 *__restrict__ src, float c,
                         long long total) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) dst[i] = make_float2(src[i].x * c, src[i].y * c);
}

__global__ void h2f(float *__restrict__ d, const __half *__restrict__ s, size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) d[i] = __half2float(s[i]);
}
__global__ void f2h(__half *__restrict__ d, const float *__restrict__ s, size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) d[i] = __float2half_rn(s[i]);
}

// ---- own-FFT convolution ------------------------------------------------------
constexpr int LC_GW = 8;

// column 0 of the filter, Hermitian part: h0[k] = (f[k][0] + conj(f[-k][0])) / 2
__global__ void lc_h0(float2 *__restrict__ h0, const float2 *__restrict__ fzs, int nrho, int nc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nrho) return;
  const float2 a = fzs[(size_t)k * nc], b = fzs[(size_t)((nrho - k) % nrho) * nc];
  h0[k] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
}

// Pass 1: row r of the pair (2q, 2q + 1): forward FFT along theta of a + i b.
template <int N>
__global__ void __launch_bounds__(N / 16, (16384 / N < 16 ? 16384 / N : 16))
    lc_rows_fwd(const float *__restrict__ fl, float2 *__restrict__ t1,
                const float2 *__restrict__ tw, int nb, int nrho) {
  extern __shared__ float2 fsm[];
  const int r = blockIdx.x, q = blockIdx.y;
  const size_t img = (size_t)nrho * N;
  const float *a = fl + (size_t)(2 * q) * img + (size_t)r * N;
  const float *b = 2 * q + 1 < nb ? a + img : nullptr;
  float2 *dst = t1 + (size_t)q * nrho * N + (size_t)r * LC_GW;
  auto in = [a, b](int e) { return make_float2(__ldg(a + e), b ? -__ldg(b + e) : 0.f); };
  auto out = [dst, nrho](int o, float2 v) {
    dst[(size_t)(o / LC_GW) * nrho * LC_GW + o % LC_GW] = make_float2(v.x, -v.y);
  };
  fftk::ifft<N>(fsm, threadIdx.x, tw, in, out);
}

// Pass 2: cpc adjacent columns k2 per block: forward FFT along rho, times
// H(k1, k2) (column 0: h0; k2 <= ntheta/2: fzs; beyond: conj(fzs(-k1, -k2))),
// inverse FFT along rho, to t2[q][k1][k2].
template <int N>
__global__ void __launch_bounds__(1024)
    lc_cols(const float2 *__restrict__ t1, float2 *__restrict__ t2,
            const float2 *__restrict__ fzs, const float2 *__restrict__ h0,
            const float2 *__restrict__ tw, int ntheta, int cpc) {
  extern __shared__ float2 fsm[];
  constexpr int SSTR = fftk::Plan<N>::PADDED + 4;
  const int c = threadIdx.x % cpc, tid = threadIdx.x / cpc;
  const int ncb = ntheta / cpc;
  const int q = blockIdx.x / ncb, j = (blockIdx.x % ncb) * cpc + c;
  const int nc = ntheta / 2 + 1;
  const float2 *src = t1 + (size_t)q * N * ntheta + (size_t)(j / LC_GW) * N * LC_GW + j % LC_GW;
  float2 *sm = fsm + c * SSTR;
  auto in1 = [src](int e) {
    const float2 v = __ldg(src + (size_t)e * LC_GW);
    return make_float2(v.x, -v.y);
  };
  auto out1 = [sm](int o, float2 v) { sm[fftk::pad16(o)] = make_float2(v.x, -v.y); };
  fftk::ifft<N, true>(sm, tid, tw, in1, out1);
  __syncthreads();
  {
    const bool neg = j >= nc;
    for (int k = tid; k < N; k += N / 16) {
      float2 hv;
      if (j == 0) {
        hv = __ldg(h0 + k);
      } else if (!neg) {
        hv = __ldg(fzs + (size_t)k * nc + j);
      } else {
        const float2 t = __ldg(fzs + (size_t)((N - k) & (N - 1)) * nc + (ntheta - j));
        hv = make_float2(t.x, -t.y);
      }
      float2 &x = sm[fftk::pad16(k)];
      x = make_float2(x.x * hv.x - x.y * hv.y, x.x * hv.y + x.y * hv.x);
    }
  }
  __syncthreads();
  float2 *dst = t2 + (size_t)q * N * ntheta + j;
  auto in2 = [sm](int e) { return sm[fftk::pad16(e)]; };
  auto out2 = [dst, ntheta](int o, float2 v) { dst[(size_t)o * ntheta] = v; };
  const float2 *tw2;  // the second transform reloads its twiddles
  asm volatile("mov.b64 %0, %1;" : "=l"(tw2) : "l"(tw));
  fftk::ifft<N>(sm, tid, tw2, in2, out2);
}

// Pass 3: row r: inverse FFT along theta, real part to slice 2q, imaginary
// part to slice 2q + 1.
template <int N>
__global__ void __launch_bounds__(N / 16, (16384 / N < 16 ? 16384 / N : 16))
    lc_rows_inv(const float2 *__restrict__ t2, float *__restrict__ fl,
                const float2 *__restrict__ tw, int nb, int nrho) {
  extern __shared__ float2 fsm[];
  const int r = blockIdx.x, q = blockIdx.y;
  const size_t img = (size_t)nrho * N;
  const float2 *src = t2 + ((size_t)q * nrho + r) * N;
  float *a = fl + (size_t)(2 * q) * img + (size_t)r * N;
  float *b = 2 * q + 1 < nb ? a + img : nullptr;
  auto in = [src](int e) { return __ldg(src + e); };
  auto out = [a, b](int o, float2 v) {
    a[o] = v.x;
    if (b) b[o] = v.y;
  };
  fftk::ifft<N>(fsm, threadIdx.x, tw, in, out);
}

inline int lc_cpc(int N) { return std::min(16384 / N, 16); }
inline size_t lc_cols_smem(int N) { return (size_t)lc_cpc(N) * (N + N / 16 + 4) * sizeof(float2); }
inline size_t lc_rows_smem(int N) { return (size_t)(N + N / 16) * sizeof(float2); }

#define LC_DISPATCH(n, F)      \
  switch (n) {                 \
    case 256: F(256); break;   \
    case 512: F(512); break;   \
    case 1024: F(1024); break; \
    case 2048: F(2048); break; \
    case 4096: F(4096); break; \
    default: F(8192); break;   \
  }

cudaError_t lc_attrs(int nrho, int ntheta) {
  cudaError_t e = cudaSuccess;
#define LC_ROWS_ATTR(N)                                                                 \
  e = cudaFuncSetAttribute(lc_rows_fwd<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                           (int)lc_rows_smem(N));                                       \
  if (e == cudaSuccess)                                                                 \
    e = cudaFuncSetAttribute(lc_rows_inv<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             (int)lc_rows_smem(N));
#define LC_COLS_ATTR(N)                                                                 \
  e = cudaFuncSetAttribute(lc_cols<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                           (int)lc_cols_smem(N));
  LC_DISPATCH(ntheta, LC_ROWS_ATTR)
  if (e != cudaSuccess) return e;
  LC_DISPATCH(nrho, LC_COLS_ATTR)
#undef LC_ROWS_ATTR
#undef LC_COLS_ATTR
  return e;
}

int lc_apply(tcb_lprec *h, cudaStream_t s) {
  const int nrho = h->nrho, ntheta = h->ntheta, nb = h->nz;
  const unsigned pairs = (unsigned)((nb + 1) / 2);
#define LC_FWD(N)                                                                      \
  lc_rows_fwd<N><<<dim3((unsigned)nrho, pairs), N / 16, lc_rows_smem(N), s>>>(h->fl, h->t1, \
                                                                            h->twt, nb, nrho)
  LC_DISPATCH(ntheta, LC_FWD)
#undef LC_FWD
  TCB_LAUNCH_CHECK();
#define LC_COLS(N)                                                                     \
  lc_cols<N><<<(unsigned)(ntheta / lc_cpc(N)) * pairs, lc_cpc(N) * (N / 16), lc_cols_smem(N), \
               s>>>(h->t1, h->t2, h->fzs, h->h0, h->twr, ntheta, lc_cpc(N))
  LC_DISPATCH(nrho, LC_COLS)
#undef LC_COLS
  TCB_LAUNCH_CHECK();
#define LC_INV(N)                                                                      \
  lc_rows_inv<N><<<dim3((unsigned)nrho, pairs), N / 16, lc_rows_smem(N), s>>>(h->t2, h->fl, \
                                                                            h->twt, nb, nrho)
  LC_DISPATCH(ntheta, LC_INV)
#undef LC_INV
  TCB_LAUNCH_CHECK();
  count_launch(3);
  return TCB_OK;
}

bool lc_pow2(int n) { return n >= 256 && n <= 8192 && (n & (n - 1)) == 0; }

int copy_to_array(cudaArray_t arr, const float *src, int w, int h, int d, cudaStream_t s) {
  cudaMemcpy3DParms p = {};
  p.srcPtr = make_cudaPitchedPtr((void *)src, w * sizeof(float), w, h);
  p.dstArray = arr;
  p.kind = cudaMemcpyDeviceToDevice;
  p.extent = make_cudaExtent(w, h, d);
  TCB_CUDA(cudaMemcpy3DAsync(&p, s));
  return TCB_OK;
}

void release(tcb_lprec *h) {
  if (h->fwd) cufftDestroy(h->fwd);
  if (h->inv) cufftDestroy(h->inv);
  if (h->texg) cudaDestroyTextureObject(h->texg);
  if (h->texfl) cudaDestroyTextureObject(h->texfl);
  if (h->ga) cudaFreeArray(h->ga);
  if (h->fla) cudaFreeArray(h->fla);
  cudaFree(h->fzs);
  cudaFree(h->fl);
  cudaFree(h->flc);
  cudaFree(h->g32);
  cudaFree(h->f32);
  cudaFree(h->t1);
  cudaFree(h->t2);
  cudaFree(h->h0);
  cudaFree(h->twr);
  cudaFree(h->twt);
  h->t1 = h->t2 = h->h0 = h->twr = h->twt = nullptr;
  h->fwd = h->inv = 0;
  h->texg = h->texfl = 0;
  h->ga = h->fla = nullptr;
  h->fzs = nullptr;
  h->fl = h->g32 = h->f32 = nullptr;
  h->flc = nullptr;
}

int make_tex(cudaArray_t arr, cudaTextureObject_t *tex) {
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = cudaAddressModeWrap;
  td.addressMode[1] = cudaAddressModeWrap;
  td.filterMode = cudaFilterModeLinear;
  td.normalizedCoords = 1;
  td.readMode = cudaReadModeElementType;
  TCB_CUDA(cudaCreateTextureObject(tex, &rd, &td, nullptr));
  return TCB_OK;
}

}  // namespace lp
}  // namespace tcb

using namespace tcb;
using namespace tcb::lp;

extern "C" int tcb_lprec_create(tcb_lprec **out, size_t nproj, size_t nz, size_t n,
                                size_t ntheta, size_t nrho, int precision) {
  TCB_CHECK_ARG(out, "tcb_lprec_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 2 && nz >= 1 && n >= 2 && ntheta >= 2 && nrho >= 2 &&
                    ntheta % 2 == 0,
                "tcb_lprec_create: bad sizes");
  TCB_CHECK_ARG(nz < 2048 && n < 65536 && nproj < 65536, "tcb_lprec_create: sizes too large");
  TCB_CHECK_ARG(precision == TCB_FLOAT32 || precision == TCB_FLOAT16,
                "tcb_lprec_create: bad precision %d", precision);
  tcb_lprec *h = new tcb_lprec();
  h->nproj = (int)nproj;
  h->nz = (int)nz;
  h->n = (int)n;
  h->ntheta = (int)ntheta;
  h->nrho = (int)nrho;
  h->precision = precision;
  auto fail = [&](int code, const char *what) {
    if (what) set_error("tcb_lprec_create: %s", what);
    release(h);
    delete h;
    return code;
  };
  size_t nc = ntheta / 2 + 1;
  if (cudaMalloc(&h->fl, nz * ntheta * nrho * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->flc, nz * nc * nrho * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&h->fzs, nc * nrho * sizeof(float2)) != cudaSuccess)
    return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  if (precision == TCB_FLOAT16 &&
      (cudaMalloc(&h->g32, nz * nproj * n * sizeof(float)) != cudaSuccess ||
       cudaMalloc(&h->f32, nz * n * n * sizeof(float)) != cudaSuccess))
    return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
  if (cudaMalloc3DArray(&h->ga, &cd, make_cudaExtent(n, nproj, nz), cudaArrayLayered) !=
          cudaSuccess ||
      cudaMalloc3DArray(&h->fla, &cd, make_cudaExtent(ntheta, nrho, nz), cudaArrayLayered) !=
          cudaSuccess)
    return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc3DArray failed");
  if (make_tex(h->ga, &h->texg) != TCB_OK || make_tex(h->fla, &h->texfl) != TCB_OK)
    return fail(TCB_ERR_CUDA, nullptr);
  int dims[2] = {(int)nrho, (int)ntheta};
  int cemb[2] = {(int)nrho, (int)nc};
  if (cufftPlanMany(&h->fwd, 2, dims, dims, 1, (int)(nrho * ntheta), cemb, 1,
                    (int)(nrho * nc), CUFFT_R2C, (int)nz) != CUFFT_SUCCESS ||
      cufftPlanMany(&h->inv, 2, dims, cemb, 1, (int)(nrho * nc), dims, 1,
                    (int)(nrho * ntheta), CUFFT_C2R, (int)nz) != CUFFT_SUCCESS)
    return fail(TCB_ERR_CUFFT, "cufftPlanMany failed");
  h->own = lc_pow2((int)nrho) && lc_pow2((int)ntheta) && std::getenv("TCB_LPREC_FFT") == nullptr;
  if (h->own) {
    const size_t pairs = (nz + 1) / 2;
    const std::vector<float2> tr = fftk::twiddle_table((int)nrho), tt = fftk::twiddle_table((int)ntheta);
    if (cudaMalloc(&h->t1, pairs * nrho * ntheta * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&h->t2, pairs * nrho * ntheta * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&h->h0, nrho * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&h->twr, tr.size() * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&h->twt, tt.size() * sizeof(float2)) != cudaSuccess)
      return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    if (cudaMemcpy(h->twr, tr.data(), tr.size() * sizeof(float2), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(h->twt, tt.data(), tt.size() * sizeof(float2), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        lc_attrs((int)nrho, (int)ntheta) != cudaSuccess)
      return fail(TCB_ERR_CUDA, "own-FFT setup failed");
  }
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_lprec_setgrids(tcb_lprec *h, const void *fz, const float *lp2p1,
                                  const float *lp2p2, const float *lp2p1w, const float *lp2p2w,
                                  const float *C2lp1, const float *C2lp2, const int *lpids,
                                  const int *wids, const int *cids, size_t nlpids,
                                  size_t nwids, size_t ncids) {
  TCB_CHECK_ARG(h && h->fl, "tcb_lprec_setgrids: null or freed handle");
  TCB_CHECK_ARG(fz && lp2p1 && lp2p2 && C2lp1 && C2lp2 && lpids && cids,
                "tcb_lprec_setgrids: null pointer");
  TCB_CHECK_ARG(nwids == 0 || (lp2p1w && lp2p2w && wids), "tcb_lprec_setgrids: null wrap grid");
  TCB_CHECK_ARG(nlpids < (1u << 31) && nwids < (1u << 31) && ncids < (1u << 31),
                "tcb_lprec_setgrids: too many points");
  h->fz = (const float2 *)fz;
  h->lp2p1 = lp2p1;
  h->lp2p2 = lp2p2;
  h->lp2p1w = lp2p1w;
  h->lp2p2w = lp2p2w;
  h->C2lp1 = C2lp1;
  h->C2lp2 = C2lp2;
  h->lpids = lpids;
  h->wids = wids;
  h->cids = cids;
  h->nlpids = (int)nlpids;
  h->nwids = (int)nwids;
  h->ncids = (int)ncids;
  long long total = (long long)(h->ntheta / 2 + 1) * h->nrho;
  scale_fz<<<ceil_div(total, 256), 256>>>(h->fzs, h->fz, 2 / (float)(h->nrho * h->ntheta),
                                          total);
  TCB_LAUNCH_CHECK();
  if (h->own) {
    lc_h0<<<ceil_div(h->nrho, 256), 256>>>(h->h0, h->fzs, h->nrho, h->ntheta / 2 + 1);
    TCB_LAUNCH_CHECK();
  }
  TCB_CUDA(cudaDeviceSynchronize());
  return TCB_OK;
}

// cfunc_lprec::backprojection: f [nz, n, n] = lprec(g [nz, nproj, n]); g is
// overwritten by its B-spline coefficients, as in the reference.
extern "C" int tcb_lprec_backprojection(tcb_lprec *h, void *f, void *g, void *stream) {
  TCB_CHECK_ARG(h && h->fl, "tcb_lprec_backprojection: null or freed handle");
  TCB_CHECK_ARG(f && g, "tcb_lprec_backprojection: null pointer");
  TCB_CHECK_ARG(h->fz, "tcb_lprec_backprojection: setgrids was not called");
  cudaStream_t s = (cudaStream_t)stream;
  const int n = h->n, nproj = h->nproj, nz = h->nz, ntheta = h->ntheta, nrho = h->nrho;
  float *gf = (float *)g, *ff = (float *)f;
  size_t gtot = (size_t)nz * nproj * n, ftot = (size_t)nz * n * n;
  if (h->precision == TCB_FLOAT16) {
    h2f<<<ceil_div(gtot, 256), 256, 0, s>>>(h->g32, (const __half *)g, gtot);
    TCB_LAUNCH_CHECK();
    count_launch();
    gf = h->g32;
    ff = h->f32;
  }
  TCB_CUDA(cudaMemsetAsync(ff, 0, ftot * sizeof(float), s));
  {
    StageTimer st("lprec_prefilter", s);
    long long nrows = (long long)nz * nproj;
    prefilter_rows<<<ceil_div(nrows, 256), 256, 0, s>>>(gf, n, nrows);
    TCB_LAUNCH_CHECK();
    dim3 grd(ceil_div(n, 128), nz);
    prefilter_cols<<<grd, 128, 0, s>>>(gf, n, nproj, nz);
    TCB_LAUNCH_CHECK();
    count_launch(2);
  }
  if (copy_to_array(h->ga, gf, n, nproj, nz, s) != TCB_OK) return TCB_ERR_CUDA;
  TCB_CUFFT(cufftSetStream(h->fwd, s));
  TCB_CUFFT(cufftSetStream(h->inv, s));
  long long lpstep = (long long)ntheta * nrho;
  long long nc = (long long)(ntheta / 2 + 1) * nrho;
  for (int k = 0; k < 3; k++) {
    TCB_CUDA(cudaMemsetAsync(h->fl, 0, (size_t)nz * lpstep * sizeof(float), s));
    {
      StageTimer st("lprec_interp_lp", s);
      dim3 g1(ceil_div(h->nlpids, 256), nz);
      interp_points<<<g1, 256, 0, s>>>(h->texg, h->fl, h->lp2p2 + (size_t)k * h->nlpids,
                                       h->lp2p1 + (size_t)k * h->nlpids, h->nlpids, n, nproj,
                                       h->lpids, lpstep);
      TCB_LAUNCH_CHECK();
      count_launch();
      if (h->nwids > 0) {
        dim3 g2(ceil_div(h->nwids, 256), nz);
        interp_points<<<g2, 256, 0, s>>>(h->texg, h->fl, h->lp2p2w + (size_t)k * h->nwids,
                                         h->lp2p1w + (size_t)k * h->nwids, h->nwids, n, nproj,
                                         h->wids, lpstep);
        TCB_LAUNCH_CHECK();
        count_launch();
      }
    }
    if (h->own) {
      StageTimer st("lprec_fft", s);
      const int rc = lc_apply(h, s);
      if (rc != TCB_OK) return rc;
    } else {
      StageTimer st("lprec_fft", s);
      TCB_CUFFT(cufftExecR2C(h->fwd, h->fl, (cufftComplex *)h->flc));
      mul_fz<<<ceil_div(nc * nz, 256), 256, 0, s>>>(h->flc, h->fzs, nc, nc * nz);
      TCB_LAUNCH_CHECK();
      count_launch();
      TCB_CUFFT(cufftExecC2R(h->inv, (cufftComplex *)h->flc, h->fl));
    }
    if (copy_to_array(h->fla, h->fl, ntheta, nrho, nz, s) != TCB_OK) return TCB_ERR_CUDA;
    {
      StageTimer st("lprec_interp_c", s);
      dim3 g4(ceil_div(h->ncids, 256), nz);
      interp_points<<<g4, 256, 0, s>>>(h->texfl, ff, h->C2lp1 + (size_t)k * h->ncids,
                                       h->C2lp2 + (size_t)k * h->ncids, h->ncids, ntheta, nrho,
                                       h->cids, (long long)n * n);
      TCB_LAUNCH_CHECK();
      count_launch();
    }
  }
  if (h->precision == TCB_FLOAT16) {
    f2h<<<ceil_div(ftot, 256), 256, 0, s>>>((__half *)f, h->f32, ftot);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

extern "C" int tcb_lprec_destroy(tcb_lprec *h) {
  if (!h) return TCB_OK;
  release(h);
  delete h;
  return TCB_OK;
}
