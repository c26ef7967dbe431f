// Fourier-gridding (USFFT) backprojector for parallel-beam tomography.
//
// Same algorithm and constants as cfunc_fourierrec (src/cuda/cfunc_fourierrec.cu,
// src/include/kernels_fourierrec.cuh): 1D FFT of each projection, Gaussian
// gridding of the polar samples onto a 2x oversampled Cartesian grid
// (eps = 1e-3, half-width m = 4), 2D inverse FFT, deapodization, circular mask.
//
// B200 design (this is not a transcription of the reference kernels):
//  * ifftshiftc before/after the 1D FFT becomes an index shift by n/2 plus a
//    (-1)^k sign at read time, so g is transformed in a single cuFFT call.
//  * The gridding kernel is tile-stationary: each CTA owns a T x T tile of the
//    periodic (2n)^2 grid, finds the polar samples whose (2m+1)^2 footprint
//    touches the tile (an analytic radial interval per angle), accumulates
//    them in shared memory and writes the finished tile once.  No global
//    atomics, no memset of the grid, the halo "wrap" pass disappears (the
//    grid is periodic by construction) and the fftshift sign before the 2D
//    FFT is applied in the store.  Tiles are dispatched centre-first because
//    the polar sample density (and so the work per tile) peaks at the origin.
//  * The 2D FFT runs on a dense (2n)^2 grid; the fftshift after it, divphi,
//    circ and (optionally) the real/imaginary unpacking of the slice pairs
//    are one kernel.
// Sample positions use the same intrinsics and operation order as takexy
// (kernels_fourierrec.cuh:23-36), so the footprint of every sample is the
// one the reference scatters to.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

#define TCB_PI_F 3.1415926535f

namespace tcb {
namespace fr {

constexpr int M = 4;          // gridding half-width for eps = 1e-3 (any n)
constexpr int T = 64;         // grid tile edge
constexpr int NT = 256;       // threads per gridding CTA
constexpr int CHUNK = NT;     // angles enumerated per pass
constexpr int MAXSEG = 4 * CHUNK;
// Margin of the ell/(2n) table: __cosf/__sinf may exceed 1 in magnitude by an
// ulp, which moves floor(2n*x0) one cell below -n.
constexpr int EPAD = 8;

struct Geom {
  int n, nproj, nz;
  int twon;        // 2n (grid edge)
  int ntx;         // tiles per grid edge
  float mu, coeff0, coeff1, scale;
};

// cos/sin of every angle with the reference's intrinsics, the radial
// coordinate table r_i = (i - n/2)/n and the grid coordinate table
// ell/(2n) for ell in [-n-m-EPAD, n+m+EPAD].
__global__ void setup_tables(float2 *__restrict__ cs, float *__restrict__ rtab,
                             float *__restrict__ etab, const float *__restrict__ theta,
                             int n, int nproj) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nproj) cs[t] = make_float2(__cosf(theta[t]), __sinf(theta[t]));
  if (t < n) rtab[t] = (t - n / 2) / (float)n;
  if (t < 2 * n + 2 * M + 1 + 2 * EPAD) {
    int ell = t - n - M - EPAD;
    etab[t] = ell / (float)(2 * n);
  }
}

// Interval of u with u*c in [a, b] (u unbounded when c ~ 0 and 0 in [a, b]).
__device__ __forceinline__ void u_interval(float c, float a, float b, float &lo, float &hi) {
  if (fabsf(c) < 1e-12f) {
    if (a <= 0.f && 0.f <= b) {
      lo = -3.0e38f;
      hi = 3.0e38f;
    } else {
      lo = 1.f;
      hi = -1.f;
    }
    return;
  }
  float u0 = a / c, u1 = b / c;
  lo = fminf(u0, u1);
  hi = fmaxf(u0, u1);
}

// Block-wide exclusive scan of one int per thread (NT threads).
__device__ __forceinline__ int block_exscan(int v, int *warp_tot, int &total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = (lane < NT / 32) ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < NT / 32) warp_tot[lane] = t;  // inclusive prefix of warp totals
  }
  __syncthreads();
  int base = wid > 0 ? warp_tot[wid - 1] : 0;
  total = warp_tot[NT / 32 - 1];
  __syncthreads();
  return base + x - v;
}

struct GatherSmem {
  // rows padded to T+1 floats: lanes that walk a near-vertical line of
  // samples hit rows two apart, which with a stride of T (a multiple of the 32
  // banks) would all fall into one bank
  float accr[T][T + 1];
  float acci[T][T + 1];
  int seg_p[MAXSEG];     // angle | image << 20
  int seg_i0[MAXSEG];
  int seg_start[MAXSEG + 1];
  int warp_tot[NT / 32];
};

// Gridding of the polar spectrum onto the periodic (2n)^2 grid.
//   G: [nz, nproj, n] complex, plain forward FFT of each projection
//   grid: [nz, 2n, 2n] complex, output (fftshift sign included)
__global__ void __launch_bounds__(NT) gather_tiles(const float2 *__restrict__ G,
                                                   float2 *__restrict__ grid,
                                                   const float2 *__restrict__ cs,
                                                   const float *__restrict__ rtab,
                                                   const float *__restrict__ etab,
                                                   const int *__restrict__ tile_order,
                                                   Geom geo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GatherSmem &sm = *reinterpret_cast<GatherSmem *>(smem_raw);
  const int n = geo.n, twon = geo.twon, nproj = geo.nproj;
  const int z = blockIdx.x % geo.nz;
  const int tile = tile_order[blockIdx.x / geo.nz];
  const int ix0 = (tile % geo.ntx) * T, iy0 = (tile / geo.ntx) * T;
  const int tw = min(T, twon - ix0), th = min(T, twon - iy0);
  // centred cell coordinates of the tile: X = ix - n
  const int X0 = ix0 - n, Y0 = iy0 - n;

  for (int k = threadIdx.x; k < T * (T + 1); k += NT) {
    (&sm.accr[0][0])[k] = 0.f;
    (&sm.acci[0][0])[k] = 0.f;
  }

  // Periodic images of the sample footprint that can reach this tile.
  int kx_lo = 1, kx_hi = -1, ky_lo = 1, ky_hi = -1;
  for (int k = -1; k <= 1; k++) {
    // footprint cells ell in [fx-M, fx+M], fx in [-n, n-1]; ell + 2n*k in tile
    int lo = X0 - 2 * n * k, hi = X0 + tw - 1 - 2 * n * k;
    if (hi >= -n - M && lo <= n - 1 + M) { kx_lo = min(kx_lo, k); kx_hi = max(kx_hi, k); }
    lo = Y0 - 2 * n * k; hi = Y0 + th - 1 - 2 * n * k;
    if (hi >= -n - M && lo <= n - 1 + M) { ky_lo = min(ky_lo, k); ky_hi = max(ky_hi, k); }
  }

  const float2 *Gz = G + (size_t)z * nproj * n;
  const float twonf = (float)(2 * n);
  const int half = n / 2;

  for (int pc = 0; pc < nproj; pc += CHUNK) {
    // ---- enumerate (angle, image) segments of candidate samples ----
    int p = pc + threadIdx.x;
    int my_i0[4], my_len[4], my_img[4];
    int nseg = 0, ncand = 0;
    if (p < nproj) {
      float2 csp = cs[p];
      for (int ky = ky_lo; ky <= ky_hi; ky++)
        for (int kx = kx_lo; kx <= kx_hi; kx++) {
          float ax = (float)(X0 - M - 2 * n * kx - 2), bx = (float)(X0 + tw - 1 + M - 2 * n * kx + 2);
          float ay = (float)(Y0 - M - 2 * n * ky - 2), by = (float)(Y0 + th - 1 + M - 2 * n * ky + 2);
          float lo0, hi0, lo1, hi1;
          u_interval(csp.x, ax, bx, lo0, hi0);   // fx ~ u*cos
          u_interval(-csp.y, ay, by, lo1, hi1);  // fy ~ -u*sin
          float lo = fmaxf(lo0, lo1), hi = fminf(hi0, hi1);
          if (lo > hi) continue;
          lo = fmaxf(lo, -2.f * n);
          hi = fminf(hi, 2.f * n);
          int i0 = max(0, (int)floorf((lo + n) * 0.5f) - 1);
          int i1 = min(n - 1, (int)ceilf((hi + n) * 0.5f) + 1);
          if (i1 < i0) continue;
          my_i0[nseg] = i0;
          my_len[nseg] = i1 - i0 + 1;
          my_img[nseg] = (kx + 1) + 3 * (ky + 1);
          ncand += i1 - i0 + 1;
          nseg++;
        }
    }
    int seg_total, cand_total;
    int seg_off = block_exscan(nseg, sm.warp_tot, seg_total);
    int cand_off = block_exscan(ncand, sm.warp_tot, cand_total);
    if (cand_total == 0) continue;  // uniform across the block
    {
      int c = cand_off;
      for (int k = 0; k < nseg; k++) {
        sm.seg_p[seg_off + k] = p | (my_img[k] << 20);
        sm.seg_i0[seg_off + k] = my_i0[k];
        sm.seg_start[seg_off + k] = c;
        c += my_len[k];
      }
      if (threadIdx.x == 0) sm.seg_start[seg_total] = cand_total;
    }
    __syncthreads();

    // ---- scatter the candidates into the shared tile ----
    for (int j = threadIdx.x; j < cand_total; j += NT) {
      int lo = 0, hi = seg_total - 1;
      while (lo < hi) {  // last segment with start <= j
        int mid = (lo + hi + 1) >> 1;
        if (sm.seg_start[mid] <= j) lo = mid; else hi = mid - 1;
      }
      int pp = sm.seg_p[lo];
      int img = pp >> 20;
      int ang = pp & 0xFFFFF;
      int i = sm.seg_i0[lo] + (j - sm.seg_start[lo]);
      float2 csa = cs[ang];
      float r = rtab[i];
      // sample position exactly as takexy computes it
      float x0 = r * csa.x;
      float y0 = -(r * csa.y);
      if (x0 >= 0.5f) x0 = 0.5f - 1e-5;
      if (y0 >= 0.5f) y0 = 0.5f - 1e-5;
      int b0 = (int)floorf(twonf * x0) - M;
      int b1 = (int)floorf(twonf * y0) - M;
      int kx = img % 3 - 1, ky = img / 3 - 1;
      // tile-local coordinates of the footprint corner
      int lx0 = b0 + 2 * n * kx - X0;
      int ly0 = b1 + 2 * n * ky - Y0;
      if (lx0 > tw - 1 || lx0 + 2 * M < 0 || ly0 > th - 1 || ly0 + 2 * M < 0) continue;
      // spectrum value with the ifftshift pair folded in: (-1)^i G[(i+n/2) mod n]
      int ii = i + half;
      if (ii >= n) ii -= n;
      float2 gv = Gz[(size_t)ang * n + ii];
      float sg = (i & 1) ? -geo.scale : geo.scale;
      float gx = gv.x * sg, gy = gv.y * sg;
      float k0[2 * M + 1], k1[2 * M + 1];
#pragma unroll
      for (int t = 0; t < 2 * M + 1; t++) {
        float w0 = etab[b0 + t + n + M + EPAD] - x0;
        k0[t] = __expf(geo.coeff1 * w0 * w0);
        float w1 = etab[b1 + t + n + M + EPAD] - y0;
        k1[t] = __expf(geo.coeff1 * w1 * w1);
      }
      if (lx0 >= 0 && lx0 + 2 * M < tw && ly0 >= 0 && ly0 + 2 * M < th) {
#pragma unroll
        for (int t1 = 0; t1 < 2 * M + 1; t1++) {
#pragma unroll
          for (int t0 = 0; t0 < 2 * M + 1; t0++) {
            float w = geo.coeff0 * (k0[t0] * k1[t1]);
            atomicAdd(&sm.accr[ly0 + t1][lx0 + t0], w * gx);
            atomicAdd(&sm.acci[ly0 + t1][lx0 + t0], w * gy);
          }
        }
      } else {
#pragma unroll
        for (int t1 = 0; t1 < 2 * M + 1; t1++) {
          int ly = ly0 + t1;
          if (ly < 0 || ly >= th) continue;
#pragma unroll
          for (int t0 = 0; t0 < 2 * M + 1; t0++) {
            int lx = lx0 + t0;
            if (lx < 0 || lx >= tw) continue;
            float w = geo.coeff0 * (k0[t0] * k1[t1]);
            atomicAdd(&sm.accr[ly][lx], w * gx);
            atomicAdd(&sm.acci[ly][lx], w * gy);
          }
        }
      }
    }
    __syncthreads();
  }

  // ---- store the tile with the pre-FFT fftshift sign ----
  float2 *gz = grid + (size_t)z * twon * twon;
  for (int k = threadIdx.x; k < T * T; k += NT) {
    int ly = k / T, lx = k % T;
    if (ly >= th || lx >= tw) continue;
    int ix = ix0 + lx, iy = iy0 + ly;
    // sign of fftshiftc on the (2n+2m)^2 buffer at index (ix+m, iy+m)
    int sx = 1 - 2 * ((ix + M + 1) % 2), sy = 1 - 2 * ((iy + M + 1) % 2);
    float sgn = (float)(sx * sy);
    gz[(size_t)iy * twon + ix] = make_float2(sm.accr[ly][lx] * sgn, sm.acci[ly][lx] * sgn);
  }
}

// fftshift after the 2D FFT + divphi + circ (+ optional unpacking).
//   grid: [nz, 2n, 2n]; f complex [nz, n, n] (unpack == 0) or
//   f real [2nz, n, n] (unpack == 1).
template <typename OutT>
__global__ void deapod_kernel(const float2 *__restrict__ grid, OutT *__restrict__ f,
                              Geom geo, int unpack) {
  const int n = geo.n, twon = geo.twon;
  int tx = blockIdx.x * blockDim.x + threadIdx.x;
  int ty = blockIdx.y * blockDim.y + threadIdx.y;
  int tz = blockIdx.z;
  if (tx >= n || ty >= n) return;
  int ix = tx + n / 2, iy = ty + 1 + n / 2;
  float2 v = grid[(size_t)tz * twon * twon + (size_t)iy * twon + ix];
  int sx = 1 - 2 * ((ix + M + 1) % 2), sy = 1 - 2 * ((iy + M + 1) % 2);
  float sgn = (float)(sx * sy);
  v.x *= sgn;
  v.y *= sgn;
  float dx = tx / (float)n - 0.5;
  float dy = ty / (float)n - 0.5;
  float phi = __expf(geo.mu * (n * n) * (dx * dx + dy * dy)) / geo.nproj;
  phi *= (1 - n % 4);
  v.x *= phi;
  v.y *= phi;
  float x = (tx - n / 2) / float(n);
  float y = (ty - n / 2) / float(n);
  float lam = (float)((4 * x * x + 4 * y * y) < 1);
  v.x *= lam;
  v.y *= lam;
  size_t plane = (size_t)n * n;
  size_t o = (size_t)ty * n + tx;
  if (unpack) {
    f[(size_t)tz * plane + o] = (OutT)v.x;
    f[(size_t)(tz + geo.nz) * plane + o] = (OutT)v.y;
  } else {
    f[2 * ((size_t)tz * plane + o)] = (OutT)v.x;
    f[2 * ((size_t)tz * plane + o) + 1] = (OutT)v.y;
  }
}

template <typename InT>
__global__ void pack_kernel(float2 *__restrict__ g, const InT *__restrict__ src, int nz,
                            int nproj, int n, size_t row_stride, size_t xoff) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int p = blockIdx.y;
  int z = blockIdx.z;
  if (x >= n) return;
  const InT *a = src + ((size_t)z * nproj + p) * row_stride + xoff;
  const InT *b = src + ((size_t)(z + nz) * nproj + p) * row_stride + xoff;
  g[((size_t)z * nproj + p) * n + x] = make_float2((float)a[x], (float)b[x]);
}

__global__ void half2_to_float2(float2 *__restrict__ dst, const __half2 *__restrict__ src,
                                size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) dst[i] = __half22float2(src[i]);
}

}  // namespace fr
}  // namespace tcb

struct tcb_fourierrec {
  size_t nproj, nz, n;
  int precision;
  tcb::fr::Geom geo;
  float2 *cs = nullptr;
  float *rtab = nullptr;
  float *etab = nullptr;
  int *tile_order = nullptr;
  float2 *grid = nullptr;
  float2 *g32 = nullptr;  // fp32 staging of g (FLOAT16 only)
  cufftHandle plan1d = 0, plan2d = 0;
  int ntiles = 0;
};

using namespace tcb;
using namespace tcb::fr;

namespace {

void fr_release(tcb_fourierrec *h) {
  if (h->plan1d) cufftDestroy(h->plan1d);
  if (h->plan2d) cufftDestroy(h->plan2d);
  cudaFree(h->cs);
  cudaFree(h->rtab);
  cudaFree(h->etab);
  cudaFree(h->tile_order);
  cudaFree(h->grid);
  cudaFree(h->g32);
  h->plan1d = h->plan2d = 0;
  h->cs = nullptr;
  h->rtab = h->etab = nullptr;
  h->tile_order = nullptr;
  h->grid = h->g32 = nullptr;
}

constexpr size_t kGatherSmem = sizeof(GatherSmem);

int fr_run(tcb_fourierrec *h, void *f, void *g, void *stream, int unpack) {
  TCB_CHECK_ARG(h, "fourierrec: null handle");
  TCB_CHECK_ARG(h->grid, "fourierrec: handle was freed");
  TCB_CHECK_ARG(f && g, "fourierrec: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  const Geom &geo = h->geo;
  float2 *gc = (float2 *)g;
  size_t gtotal = h->nz * h->nproj * h->n;
  if (h->precision == TCB_FLOAT16) {
    half2_to_float2<<<ceil_div(gtotal, 256), 256, 0, s>>>(h->g32, (const __half2 *)g, gtotal);
    TCB_LAUNCH_CHECK();
    count_launch();
    gc = h->g32;
  }
  TCB_CUFFT(cufftSetStream(h->plan1d, s));
  TCB_CUFFT(cufftSetStream(h->plan2d, s));
  {
    StageTimer st("fr_fft1d", s);
    TCB_CUFFT(cufftExecC2C(h->plan1d, (cufftComplex *)gc, (cufftComplex *)gc, CUFFT_FORWARD));
  }
  {
    StageTimer st("fr_gather", s);
    gather_tiles<<<(unsigned)(h->ntiles * h->nz), NT, kGatherSmem, s>>>(
        gc, h->grid, h->cs, h->rtab, h->etab, h->tile_order, geo);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  {
    StageTimer st("fr_fft2d", s);
    TCB_CUFFT(cufftExecC2C(h->plan2d, (cufftComplex *)h->grid, (cufftComplex *)h->grid,
                           CUFFT_INVERSE));
  }
  {
    StageTimer st("fr_deapod", s);
    dim3 blk(32, 8), grd(ceil_div(h->n, 32), ceil_div(h->n, 8), (unsigned)h->nz);
    if (h->precision == TCB_FLOAT16)
      deapod_kernel<__half><<<grd, blk, 0, s>>>(h->grid, (__half *)f, geo, unpack);
    else
      deapod_kernel<float><<<grd, blk, 0, s>>>(h->grid, (float *)f, geo, unpack);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

}  // namespace

extern "C" int tcb_fourierrec_create(tcb_fourierrec **out, size_t nproj, size_t nz,
                                     size_t n, const float *theta, int precision) {
  TCB_CHECK_ARG(out, "tcb_fourierrec_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(theta, "tcb_fourierrec_create: null theta");
  // n >= T keeps at most two periodic images of a footprint per grid axis
  // inside one tile (the enumeration below stores up to four segments per angle).
  TCB_CHECK_ARG(n >= (size_t)T && n % 2 == 0 && n <= 32768,
                "tcb_fourierrec_create: n=%zu must be even and in [%d, 32768]", n, T);
  TCB_CHECK_ARG(nproj >= 1 && nproj < (1u << 20), "tcb_fourierrec_create: bad nproj %zu",
                nproj);
  TCB_CHECK_ARG(nz >= 1, "tcb_fourierrec_create: nz must be >= 1");
  TCB_CHECK_ARG(nproj * nz < (1ull << 31), "tcb_fourierrec_create: nproj*nz too large");
  TCB_CHECK_ARG(precision == TCB_FLOAT32 || precision == TCB_FLOAT16,
                "tcb_fourierrec_create: bad precision %d", precision);
  // Constants exactly as the reference constructor computes them
  // (cfunc_fourierrec.cu:6-8; host float arithmetic).
  float eps = 1e-3f;
  float mu = -logf(eps) / (float)(2 * n * n);
  size_t m = (size_t)ceilf(2 * n * 1 / TCB_PI_F *
                           sqrtf(-mu * logf(eps) + (mu * n) * (mu * n) / 4));
  TCB_CHECK_ARG(m == (size_t)M, "tcb_fourierrec_create: unexpected gridding width m=%zu", m);

  tcb_fourierrec *h = new tcb_fourierrec();
  h->nproj = nproj;
  h->nz = nz;
  h->n = n;
  h->precision = precision;
  Geom &geo = h->geo;
  geo.n = (int)n;
  geo.nproj = (int)nproj;
  geo.nz = (int)nz;
  geo.twon = (int)(2 * n);
  geo.ntx = (int)ceil_div(2 * n, T);
  geo.mu = mu;
  geo.coeff0 = TCB_PI_F / (mu * (4 * n * n));
  geo.coeff1 = -TCB_PI_F * TCB_PI_F / mu;
  geo.scale = 4.0f / n;
  h->ntiles = geo.ntx * geo.ntx;

  auto fail = [&](int code) {
    fr_release(h);
    delete h;
    return code;
  };
#define FR_ALLOC(ptr, bytes)                                                       \
  do {                                                                             \
    cudaError_t _e = cudaMalloc((void **)&(ptr), (bytes));                         \
    if (_e != cudaSuccess) {                                                       \
      set_error("tcb_fourierrec_create: cudaMalloc(%zu) failed: %s", (size_t)(bytes), \
                cudaGetErrorString(_e));                                           \
      return fail(TCB_ERR_OUT_OF_MEMORY);                                          \
    }                                                                              \
  } while (0)
  FR_ALLOC(h->cs, nproj * sizeof(float2));
  FR_ALLOC(h->rtab, n * sizeof(float));
  FR_ALLOC(h->etab, (2 * n + 2 * M + 1 + 2 * EPAD) * sizeof(float));
  FR_ALLOC(h->tile_order, h->ntiles * sizeof(int));
  FR_ALLOC(h->grid, nz * 4 * n * n * sizeof(float2));
  if (precision == TCB_FLOAT16) FR_ALLOC(h->g32, nz * nproj * n * sizeof(float2));
#undef FR_ALLOC

  // Tiles ordered by distance of their centre from the grid origin.
  std::vector<int> order(h->ntiles);
  std::vector<float> dist(h->ntiles);
  for (int t = 0; t < h->ntiles; t++) {
    order[t] = t;
    float cx = (t % geo.ntx) * T + 0.5f * T - (float)n;
    float cy = (t / geo.ntx) * T + 0.5f * T - (float)n;
    dist[t] = cx * cx + cy * cy;
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return dist[a] < dist[b]; });
  cudaError_t e = cudaMemcpy(h->tile_order, order.data(), h->ntiles * sizeof(int),
                             cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    set_error("tcb_fourierrec_create: cudaMemcpy failed: %s", cudaGetErrorString(e));
    return fail(TCB_ERR_CUDA);
  }
  int tab = (int)std::max(std::max(nproj, n), 2 * n + 2 * M + 1 + 2 * EPAD);
  setup_tables<<<ceil_div(tab, 256), 256>>>(h->cs, h->rtab, h->etab, theta, (int)n,
                                            (int)nproj);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_error("tcb_fourierrec_create: table setup failed: %s", cudaGetErrorString(e));
    return fail(TCB_ERR_CUDA);
  }
  e = cudaFuncSetAttribute(gather_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kGatherSmem);
  if (e != cudaSuccess) {
    set_error("tcb_fourierrec_create: smem attribute failed: %s", cudaGetErrorString(e));
    return fail(TCB_ERR_CUDA);
  }
  int len1[1] = {(int)n};
  cufftResult r = cufftPlanMany(&h->plan1d, 1, len1, nullptr, 1, 0, nullptr, 1, 0,
                                CUFFT_C2C, (int)(nproj * nz));
  int len2[2] = {(int)(2 * n), (int)(2 * n)};
  if (r == CUFFT_SUCCESS)
    r = cufftPlanMany(&h->plan2d, 2, len2, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, (int)nz);
  if (r != CUFFT_SUCCESS) {
    set_error("tcb_fourierrec_create: cufftPlanMany failed: %d", (int)r);
    return fail(r == CUFFT_ALLOC_FAILED ? TCB_ERR_OUT_OF_MEMORY : TCB_ERR_CUFFT);
  }
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_fourierrec_backprojection(tcb_fourierrec *h, void *f, void *g,
                                             void *stream) {
  return fr_run(h, f, g, stream, 0);
}

extern "C" int tcb_fourierrec_backprojection_slices(tcb_fourierrec *h, void *f, void *g,
                                                    void *stream) {
  return fr_run(h, f, g, stream, 1);
}

extern "C" int tcb_fourierrec_pack(tcb_fourierrec *h, void *g, const void *src,
                                   size_t row_stride, size_t xoff, void *stream) {
  TCB_CHECK_ARG(h && g && src, "tcb_fourierrec_pack: null pointer");
  TCB_CHECK_ARG(h->grid, "tcb_fourierrec_pack: handle was freed");
  TCB_CHECK_ARG(row_stride >= xoff + h->n, "tcb_fourierrec_pack: row_stride too small");
  TCB_CHECK_ARG(h->precision == TCB_FLOAT32, "tcb_fourierrec_pack: FLOAT32 handles only");
  TCB_CHECK_ARG(h->nproj < 65536 && h->nz < 65536, "tcb_fourierrec_pack: grid too large");
  cudaStream_t s = (cudaStream_t)stream;
  dim3 grd(ceil_div(h->n, 256), (unsigned)h->nproj, (unsigned)h->nz);
  StageTimer st("fr_pack", s);
  pack_kernel<float><<<grd, 256, 0, s>>>((float2 *)g, (const float *)src, (int)h->nz,
                                         (int)h->nproj, (int)h->n, row_stride, xoff);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

extern "C" int tcb_fourierrec_destroy(tcb_fourierrec *h) {
  if (!h) return TCB_OK;
  fr_release(h);
  delete h;
  return TCB_OK;
}
