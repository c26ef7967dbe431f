// Laminography Fourier chain: 2D R2C FFT of filtered projections (fft2d),
// adjoint 2D USFFT onto each frequency row's (2n1 x 2n0) grid (usfft2d), and
// adjoint 1D USFFT along the height (usfft1d).
//
// Same transforms, constants and index conventions as the reference
// operators (src/cuda/cfunc_fft2d.cu, cfunc_usfft2d.cu, cfunc_usfft1d.cu and
// src/include/kernels_*.cu):
//  * fft2d: (-1)^(x+y) sign, R2C over (deth, detw), -(-1)^(kx+ky) sign,
//    1/(deth*detw);
//  * usfft2d adj: sample (ku, kv) of each angle sits at
//    x = ku cos(t) + kv sin(t) cos(phi), y = ku sin(t) - kv cos(t) cos(phi),
//    clamped to +-(0.5-1e-5); columns right of detw/2 use the conjugate of
//    the mirrored sample; Gaussian gridding (eps=1e-3), periodic wrap,
//    inverse 2D FFT, deapodization with the n1-ty-1 row flip;
//  * usfft1d adj: samples z = (t - deth/2)/deth sin(phi) along the height,
//    Gaussian gridding, inverse FFT along z, real part / deapodization.
//
// B200 design:
//  * usfft2d gridding is tile-stationary (one CTA per grid tile and slab,
//    samples found per angle as a parameter interval, accumulation in shared
//    memory, one store per cell): no global atomics, no memset, no wrap pass,
//    fftshift signs folded into the store and into the deapodization read.
//  * usfft1d gridding is a gather: each grid cell sums the (contiguous) run
//    of height samples that reach it, so it needs no atomics either.
//  * The fused entry points read the stage-1 spectrum of the whole dataset
//    in place (the Hermitian mirror is an index map) and write each stage's
//    output straight into the next stage's full-size array, replacing the
//    host-side packing and transposes of BackprojLamFourierParallel.
#include <cuda_fp16.h>

#include <cmath>

#include "common.cuh"

#define LAM_PI_D 3.1415926535897932384626433

namespace tcb {
namespace lam {

constexpr int T = 64;
constexpr int NT = 256;
constexpr int CHUNK = NT;
constexpr int MAXSEG = 4 * CHUNK;
constexpr int EPAD = 8;

// Gridding width/constant exactly as the reference constructors compute them.
inline void gauss_params(size_t nn, float &mu, int &m) {
  mu = (float)(-log(1e-3) / (2 * nn * nn));
  m = (int)ceil(2 * nn * 1 / LAM_PI_D * sqrt(-mu * log(1e-3) + (mu * nn) * (mu * nn) / 4));
}

__device__ __forceinline__ int sgn_idx(int t) { return 1 - 2 * ((t + 1) % 2); }

// ------------------------------------------------------------------ fft2d
__global__ void checker_real(float *__restrict__ f, int nx, int ny, size_t total) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int tx = (int)(i % nx);
  int ty = (int)((i / nx) % ny);
  f[i] *= (float)(sgn_idx(tx) * sgn_idx(ty));
}

__global__ void fft2d_post(float2 *__restrict__ g, int nxc, int ny, size_t total, float c) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int tx = (int)(i % nxc);
  int ty = (int)((i / nxc) % ny);
  float s = (float)(-(sgn_idx(tx) * sgn_idx(ty)));
  float2 v = g[i];
  v.x *= s;
  v.y *= s;
  v.x *= c;
  v.y *= c;
  g[i] = v;
}

// ------------------------------------------------------------------ usfft2d
struct U2Geom {
  int n0, n1;        // grid half-sizes (x, y); grids are 2n0 x 2n1
  int m0, m1;
  float mu0, mu1;
  int ntheta, detw, deth;   // deth = rows of this call (slabs)
  int ntx, nty;             // tiles per axis
  int k, deth0;             // chunk index and full detector height (kv)
  float wscale;             // PI / sqrt(mu0 mu1 ntheta)
  float c0, c1;             // -PI^2/mu0, -PI^2/mu1
  // sample source
  int fused;                // 0: packed [2*ntheta][deth][detw/2+1]; 1: full stage-1 array
  int row0;                 // fused: first frequency row of this call
  int deth_full;            // fused: rows of the stage-1 array
  const float *in_scale;    // fp16 storage: per-angle factor of the input (or null)
};

struct U2Smem {
  float accr[T][T + 1];  // padded rows: see the fourierrec gridding kernel
  float acci[T][T + 1];
  int seg_a[MAXSEG];
  int seg_i0[MAXSEG];
  int seg_start[MAXSEG + 1];
  int warp_tot[NT / 32];
};

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
    if (lane < NT / 32) warp_tot[lane] = t;
  }
  __syncthreads();
  int base = wid > 0 ? warp_tot[wid - 1] : 0;
  total = warp_tot[NT / 32 - 1];
  __syncthreads();
  return base + x - v;
}

__device__ __forceinline__ void interval(float c, float a, float b, float &lo, float &hi) {
  if (fabsf(c) < 1e-12f) {
    if (a <= 0.f && 0.f <= b) { lo = -3.0e38f; hi = 3.0e38f; } else { lo = 1.f; hi = -1.f; }
    return;
  }
  float u0 = a / c, u1 = b / c;
  lo = fminf(u0, u1);
  hi = fmaxf(u0, u1);
}

// Sample position as take_x computes it (kernels_usfft2d.cu:5-18); cphi is
// the device cosf(phi), as there (u2_tables stores it after the angles).  The
// roundings are written out as the reference build performs them,
// x = fma(ku, cos t, (kv sin t) cos phi) and y = fma(-(kv cos t), cos phi,
// ku sin t), so the positions are bit-identical to take_x's.
__device__ __forceinline__ void u2_pos(const U2Geom &g, float cphi, float2 csa, int tx, int ty,
                                       float &x, float &y) {
  float ku = (tx - g.detw / 2.0f) / g.detw;
  float kv = (ty + g.k * g.deth - g.deth0 / 2.0f) / g.deth0;
  x = __fmaf_rn(ku, csa.x, __fmul_rn(__fmul_rn(kv, csa.y), cphi));
  y = __fmaf_rn(-__fmul_rn(kv, csa.x), cphi, __fmul_rn(ku, csa.y));
  x = (float)fmin(fmax((double)x, -0.5f + 1e-5), 0.5f - 1e-5);
  y = (float)fmin(fmax((double)y, -0.5f + 1e-5), 0.5f - 1e-5);
}

// Storage of the stage arrays: complex fp32 (float2) or complex fp16
// (__half2, "fp16 storage"); arithmetic is fp32 either way.
__device__ __forceinline__ float2 ld2(const float2 *p) { return *p; }
__device__ __forceinline__ float2 ld2(const __half2 *p) { return __half22float2(*p); }
__device__ __forceinline__ void st2(float2 *p, float2 v) { *p = v; }
__device__ __forceinline__ void st2(__half2 *p, float2 v) { *p = __floats2half2_rn(v.x, v.y); }

// Value of sample (tx, ty, tz) with the conjugate mirror of gather2d.
template <typename S>
__device__ __forceinline__ float2 u2_val(const U2Geom &g, const S *__restrict__ src, int tx,
                                         int ty, int tz) {
  const int wc = g.detw / 2 + 1;
  if (!g.fused) {
    int txs = tx, tys = ty, tzs = tz;
    float conj = 1.f;
    if (tx > g.detw / 2) {
      txs = tx - 2 * (tx - g.detw / 2);
      tys = g.deth - ty - 1;
      tzs = tz + g.ntheta;
      conj = -1.f;
    }
    float2 v = ld2(src + (size_t)txs + (size_t)tys * wc + (size_t)tzs * wc * g.deth);
    v.y *= conj;
    return v;
  }
  const float sc = g.in_scale ? g.in_scale[tz] : 1.f;
  int row = g.row0 + ty;
  if (tx <= g.detw / 2) {
    float2 v = ld2(src + (size_t)tx + (size_t)row * wc + (size_t)tz * wc * g.deth_full);
    return make_float2(v.x * sc, v.y * sc);
  }
  int mrow = g.deth_full - row;
  if (mrow >= g.deth_full) mrow -= g.deth_full;
  float2 v = ld2(src + (size_t)(g.detw - tx) + (size_t)mrow * wc + (size_t)tz * wc * g.deth_full);
  return make_float2(v.x * sc, -v.y * sc);
}

template <int M0, int M1, typename S>
__global__ void __launch_bounds__(NT) u2_gather(const S *__restrict__ src,
                                                float2 *__restrict__ grid,
                                                const float2 *__restrict__ cs,
                                                const float *__restrict__ ex,
                                                const float *__restrict__ ey, U2Geom geo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  U2Smem &sm = *reinterpret_cast<U2Smem *>(smem_raw);
  const int n0 = geo.n0, n1 = geo.n1;
  const int ntiles = geo.ntx * geo.nty;
  const int slab = blockIdx.x / ntiles;
  const int tile = blockIdx.x % ntiles;
  const int ix0 = (tile % geo.ntx) * T, iy0 = (tile / geo.ntx) * T;
  const int tw = min(T, 2 * n0 - ix0), th = min(T, 2 * n1 - iy0);
  const int X0 = ix0 - n0, Y0 = iy0 - n1;
  for (int k = threadIdx.x; k < T * (T + 1); k += NT) {
    (&sm.accr[0][0])[k] = 0.f;
    (&sm.acci[0][0])[k] = 0.f;
  }
  int kx_lo = 1, kx_hi = -1, ky_lo = 1, ky_hi = -1;
  for (int k = -1; k <= 1; k++) {
    int lo = X0 - 2 * n0 * k, hi = X0 + tw - 1 - 2 * n0 * k;
    if (hi >= -n0 - M0 && lo <= n0 - 1 + M0) { kx_lo = min(kx_lo, k); kx_hi = max(kx_hi, k); }
    lo = Y0 - 2 * n1 * k; hi = Y0 + th - 1 - 2 * n1 * k;
    if (hi >= -n1 - M1 && lo <= n1 - 1 + M1) { ky_lo = min(ky_lo, k); ky_hi = max(ky_hi, k); }
  }
  // tiles near the grid border also receive clamped samples: no x (y) pruning there
  const bool edge_x = (X0 <= -n0 + M0 + 2) || (X0 + tw - 1 >= n0 - 1 - M0 - 2);
  const bool edge_y = (Y0 <= -n1 + M1 + 2) || (Y0 + th - 1 >= n1 - 1 - M1 - 2);
  const float kv = (slab + geo.k * geo.deth - geo.deth0 / 2.0f) / geo.deth0;
  const int detw = geo.detw;
  const float cphi = cs[geo.ntheta].x;

  for (int pc = 0; pc < geo.ntheta; pc += CHUNK) {
    int p = pc + threadIdx.x;
    int my_i0[4], my_len[4], my_img[4];
    int nseg = 0, ncand = 0;
    if (p < geo.ntheta) {
      float2 csp = cs[p];
      float ox = kv * csp.y * cphi, oy = -kv * csp.x * cphi;
      for (int ky = ky_lo; ky <= ky_hi; ky++)
        for (int kx = kx_lo; kx <= kx_hi; kx++) {
          float lo = -3.0e38f, hi = 3.0e38f, l, h;
          if (!edge_x) {
            // 2n0*(ku c + ox) in [A-2, B+2]
            float a = (float)(X0 - M0 - 2 * n0 * kx - 2) / (2.f * n0) - ox;
            float b = (float)(X0 + tw - 1 + M0 - 2 * n0 * kx + 2) / (2.f * n0) - ox;
            interval(csp.x, a, b, l, h);
            lo = fmaxf(lo, l); hi = fminf(hi, h);
          } else if (kx != 0) {
            float a = (float)(X0 - M0 - 2 * n0 * kx - 2) / (2.f * n0) - ox;
            float b = (float)(X0 + tw - 1 + M0 - 2 * n0 * kx + 2) / (2.f * n0) - ox;
            interval(csp.x, a, b, l, h);
            lo = fmaxf(lo, l); hi = fminf(hi, h);
          }
          if (!edge_y || ky != 0) {
            float a = (float)(Y0 - M1 - 2 * n1 * ky - 2) / (2.f * n1) - oy;
            float b = (float)(Y0 + th - 1 + M1 - 2 * n1 * ky + 2) / (2.f * n1) - oy;
            interval(csp.y, a, b, l, h);
            lo = fmaxf(lo, l); hi = fminf(hi, h);
          }
          if (lo > hi) continue;
          lo = fmaxf(lo, -1.f);
          hi = fminf(hi, 1.f);
          // ku = (tx - detw/2)/detw
          int i0 = max(0, (int)floorf(lo * detw + detw * 0.5f) - 1);
          int i1 = min(detw - 1, (int)ceilf(hi * detw + detw * 0.5f) + 1);
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
    if (cand_total == 0) continue;
    {
      int c = cand_off;
      for (int k = 0; k < nseg; k++) {
        sm.seg_a[seg_off + k] = p | (my_img[k] << 20);
        sm.seg_i0[seg_off + k] = my_i0[k];
        sm.seg_start[seg_off + k] = c;
        c += my_len[k];
      }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cand_total; j += NT) {
      int lo = 0, hi = seg_total - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (sm.seg_start[mid] <= j) lo = mid; else hi = mid - 1;
      }
      int a = sm.seg_a[lo];
      int img = a >> 20, ang = a & 0xFFFFF;
      int tx = sm.seg_i0[lo] + (j - sm.seg_start[lo]);
      float x0, y0;
      u2_pos(geo, cphi, cs[ang], tx, slab, x0, y0);
      int b0 = (int)floorf(2 * n0 * x0) - M0;
      int b1 = (int)floorf(2 * n1 * y0) - M1;
      int kx = img % 3 - 1, ky = img / 3 - 1;
      int lx0 = b0 + 2 * n0 * kx - X0;
      int ly0 = b1 + 2 * n1 * ky - Y0;
      if (lx0 > tw - 1 || lx0 + 2 * M0 < 0 || ly0 > th - 1 || ly0 + 2 * M1 < 0) continue;
      float2 gv = u2_val(geo, src, tx, slab, ang);
      float k0[2 * M0 + 1], k1[2 * M1 + 1];
#pragma unroll
      for (int t = 0; t < 2 * M0 + 1; t++) {
        float w0 = ex[b0 + t + n0 + M0 + EPAD] - x0;
        k0[t] = __expf(geo.c0 * (w0 * w0));
      }
#pragma unroll
      for (int t = 0; t < 2 * M1 + 1; t++) {
        float w1 = ey[b1 + t + n1 + M1 + EPAD] - y0;
        k1[t] = __expf(geo.c1 * (w1 * w1));
      }
      float gx = gv.x * geo.wscale, gy = gv.y * geo.wscale;
#pragma unroll
      for (int t1 = 0; t1 < 2 * M1 + 1; t1++) {
        int ly = ly0 + t1;
        if (ly < 0 || ly >= th) continue;
#pragma unroll
        for (int t0 = 0; t0 < 2 * M0 + 1; t0++) {
          int lx = lx0 + t0;
          if (lx < 0 || lx >= tw) continue;
          float w = k0[t0] * k1[t1];
          atomicAdd(&sm.accr[ly][lx], w * gx);
          atomicAdd(&sm.acci[ly][lx], w * gy);
        }
      }
    }
    __syncthreads();
  }
  float2 *gz = grid + (size_t)slab * (2 * n0) * (2 * n1);
  for (int k = threadIdx.x; k < T * T; k += NT) {
    int ly = k / T, lx = k % T;
    if (ly >= th || lx >= tw) continue;
    int ix = ix0 + lx, iy = iy0 + ly;
    float s = (float)(sgn_idx(ix + M0) * sgn_idx(iy + M1));
    gz[(size_t)iy * (2 * n0) + ix] = make_float2(sm.accr[ly][lx] * s, sm.acci[ly][lx] * s);
  }
}

// cs[0, ntheta): cos/sin of the angles; cs[ntheta].x: cos(phi), all with the
// device cosf/sinf that take_x calls (kernels_usfft2d.cu:14-15).
__global__ void u2_tables(float2 *__restrict__ cs, float *__restrict__ ex, float *__restrict__ ey,
                          const float *__restrict__ theta, float phi, int ntheta, int n0, int m0,
                          int n1, int m1) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ntheta) cs[t] = make_float2(cosf(theta[t]), sinf(theta[t]));
  if (t == 0) cs[ntheta] = make_float2(cosf(phi), 0.f);
  if (t < 2 * n0 + 2 * m0 + 1 + 2 * EPAD) ex[t] = (t - n0 - m0 - EPAD) / (float)(2 * n0);
  if (t < 2 * n1 + 2 * m1 + 1 + 2 * EPAD) ey[t] = (t - n1 - m1 - EPAD) / (float)(2 * n1);
}

// divker2d (direction 1) with the post-FFT fftshift sign; f[ty][slab][tx] layout
// [n1][fstride_slabs][n0], slab offset fslab0.
// fp16 storage: the output is multiplied by a power of two chosen from the
// max |grid| of this call (max_bits), so that |f| < 2^14; the inverse goes to
// out_inv[fslab0 + slab] for the consumer.
__device__ __forceinline__ float out_factor(const unsigned *max_bits, int n0, int n1) {
  if (!max_bits) return 1.f;
  // |f| <= max|grid| / ker / (n0 n1) with 1/ker < 8 (ker >= eps^(1/4))
  float bound = __uint_as_float(*max_bits) * 8.f / ((float)n0 * (float)n1);
  int e = 0;
  if (bound > 0.f) frexpf(bound, &e);
  return ldexpf(1.f, 14 - e);
}

__global__ void absmax_c(const float2 *__restrict__ g, size_t total, unsigned *__restrict__ out) {
  float m = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    float2 v = g[i];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(out, __float_as_uint(m));
}

template <typename S>
__global__ void u2_deapod(const float2 *__restrict__ grid, S *__restrict__ f, U2Geom geo,
                          int nslab, int fslabs, int fslab0, const unsigned *max_bits,
                          float *out_inv) {
  const int n0 = geo.n0, n1 = geo.n1;
  int tx = blockIdx.x * blockDim.x + threadIdx.x;
  int ty = blockIdx.y * blockDim.y + threadIdx.y;
  int tz = blockIdx.z;
  if (tx >= n0 || ty >= n1 || tz >= nslab) return;
  float ker = __expf(-geo.mu0 * (tx - n0 / 2) * (tx - n0 / 2) -
                     geo.mu1 * (ty - n1 / 2) * (ty - n1 / 2));
  int ix = tx + n0 / 2;
  int iy = n1 - ty - 1 + n1 / 2;
  float2 v = grid[(size_t)tz * (2 * n0) * (2 * n1) + (size_t)iy * (2 * n0) + ix];
  float s = (float)(sgn_idx(ix + geo.m0) * sgn_idx(iy + geo.m1));
  v.x *= s;
  v.y *= s;
  float nn = (float)(n0 * n1);
  const float of = out_factor(max_bits, n0, n1);
  if (out_inv && tx == 0 && ty == 0) out_inv[fslab0 + tz] = 1.f / of;
  st2(f + (size_t)tx + (size_t)(fslab0 + tz) * n0 + (size_t)ty * n0 * fslabs,
      make_float2(v.x / ker / nn * of, v.y / ker / nn * of));
}

// ------------------------------------------------------------------ usfft1d
struct U1Geom {
  const float *in_scale;  // fp16 storage: per-row factor of the input (or null)
  int n0, n1, n2, m2, deth;
  float mu2;
  float wscale;  // sqrt(PI / (mu2 n0))
  float c2;      // -PI^2 / mu2
};

// Gather form of gather1d(direction 1) + wrap1d + fftshiftc1d: grid cell
// (z, y, x) of the periodic [2n2][n1][n0] grid sums the height samples whose
// footprint reaches it.  g: [n1][deth/2+1][n0] (row stride gstride rows).
template <typename S>
__global__ void u1_gather(const S *__restrict__ g, float2 *__restrict__ grid,
                          const float *__restrict__ zt, const float *__restrict__ ez, U1Geom geo,
                          float zslope, float zoff) {
  const int n0 = geo.n0, n1 = geo.n1, n2 = geo.n2, M = geo.m2, deth = geo.deth;
  int tx = blockIdx.x * blockDim.x + threadIdx.x;
  int ty = blockIdx.y;
  int iz = blockIdx.z;  // periodic cell index 0..2n2-1
  if (tx >= n0) return;
  const int hc = deth / 2 + 1;
  float sr = 0.f, si = 0.f;
  // cells ell = iz - n2 + 2 n2 k (k = -1, 0, 1)
  for (int k = -1; k <= 1; k++) {
    int ell = iz - n2 + 2 * n2 * k;
    if (ell < -n2 - M - 1 || ell > n2 + M) continue;
    // samples with floor(2 n2 z) in [ell - M, ell + M]; z = zslope*t + zoff
    float a = (float)(ell - M - 2) / (2.f * n2), b = (float)(ell + M + 2) / (2.f * n2);
    int t0, t1;
    if (fabsf(zslope) < 1e-20f) {
      if (a <= zoff && zoff <= b) { t0 = 0; t1 = deth - 1; } else continue;
    } else {
      float u0 = (a - zoff) / zslope, u1 = (b - zoff) / zslope;
      t0 = max(0, (int)floorf(fminf(u0, u1)) - 1);
      t1 = min(deth - 1, (int)ceilf(fmaxf(u0, u1)) + 1);
    }
    for (int t = t0; t <= t1; t++) {
      float z0 = zt[t];
      int e0 = (int)floorf(2 * n2 * z0) - M;
      int i2 = ell - e0;
      if (i2 < 0 || i2 > 2 * M) continue;
      float w2 = ez[ell + n2 + M + EPAD] - z0;
      float w = geo.wscale * __expf(geo.c2 * (w2 * w2));
      int ts = t;
      float conj = 1.f;
      if (t > deth / 2) {
        ts = t - 2 * (t - deth / 2);
        conj = -1.f;
      }
      float2 v = ld2(g + (size_t)tx + (size_t)ts * n0 + (size_t)ty * n0 * hc);
      if (geo.in_scale) {
        v.x *= geo.in_scale[ts];
        v.y *= geo.in_scale[ts];
      }
      sr += w * v.x;
      si += w * conj * v.y;
    }
  }
  float s = (float)sgn_idx(iz + M);
  grid[(size_t)tx + (size_t)ty * n0 + (size_t)iz * n0 * n1] = make_float2(sr * s, si * s);
}

__global__ void u1_tables(float *__restrict__ zt, float *__restrict__ ez, float phi, int deth,
                          int n2, int m2) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < deth) zt[t] = (t - deth / 2.0f) / deth * sinf(phi);
  if (t < 2 * n2 + 2 * m2 + 1 + 2 * EPAD) ez[t] = (t - n2 - m2 - EPAD) / (float)(2 * n2);
}

// fftshiftc1d + divker1d(direction 1): f[ty][tz][tx] = Re / ker / (2 n2).
__global__ void u1_deapod(const float2 *__restrict__ grid, float *__restrict__ f, U1Geom geo) {
  const int n0 = geo.n0, n1 = geo.n1, n2 = geo.n2;
  int tx = blockIdx.x * blockDim.x + threadIdx.x;
  int ty = blockIdx.y;
  int tz = blockIdx.z;
  if (tx >= n0) return;
  float ker = __expf(-geo.mu2 * (tz - n2 / 2) * (tz - n2 / 2));
  int iz = tz + n2 / 2;
  float v = grid[(size_t)tx + (size_t)ty * n0 + (size_t)iz * n0 * n1].x;
  v *= (float)sgn_idx(iz + geo.m2);
  f[(size_t)tx + (size_t)tz * n0 + (size_t)ty * n0 * n2] = v / ker / (2 * n2);
}

// ------------------------------------------------------------------ forward operators
// cfunc_usfft2d::fwd (cfunc_usfft2d.cu:53-70): divker2d(direction 0) with the
// fftshift sign writes f [n1][n2 slabs][n0] / ker / (n0 n1) into the centre of
// each slab's periodic [2n1][2n0] grid (every other cell zero, so the grid
// needs no memset), a forward 2D FFT, then each sample gathers its 9 x 9
// footprint (gather2d direction 0, the fftshift sign at read time).
__global__ void u2f_load(float2 *__restrict__ grid, const float2 *__restrict__ f, U2Geom geo,
                         int nslab) {
  const int n0 = geo.n0, n1 = geo.n1;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y;
  const int slab = blockIdx.z;
  if (ix >= 2 * n0 || slab >= nslab) return;
  const int tx = ix - n0 / 2, ty = n1 - 1 + n1 / 2 - iy;
  float2 v = make_float2(0.f, 0.f);
  if (tx >= 0 && tx < n0 && ty >= 0 && ty < n1) {
    const float ker = __expf(-geo.mu0 * (tx - n0 / 2) * (tx - n0 / 2) -
                             geo.mu1 * (ty - n1 / 2) * (ty - n1 / 2));
    const float2 a = f[(size_t)tx + (size_t)slab * n0 + (size_t)ty * n0 * nslab];
    const float nn = (float)(n0 * n1);
    const float s = (float)(sgn_idx(ix + geo.m0) * sgn_idx(iy + geo.m1));
    v = make_float2(a.x / ker / nn * s, a.y / ker / nn * s);
  }
  grid[(size_t)slab * (2 * n0) * (2 * n1) + (size_t)iy * (2 * n0) + ix] = v;
}

template <int M0, int M1>
__global__ void u2f_gather(float2 *__restrict__ g, const float2 *__restrict__ grid,
                           const float2 *__restrict__ cs, const float *__restrict__ ex,
                           const float *__restrict__ ey, U2Geom geo) {
  const int n0 = geo.n0, n1 = geo.n1, detw = geo.detw, deth = geo.deth;
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y;   // detector row of this call = slab
  const int tz = blockIdx.z;   // angle
  if (tx >= detw) return;
  float x0, y0;
  u2_pos(geo, cs[geo.ntheta].x, cs[tz], tx, ty, x0, y0);
  const int b0 = (int)floorf(2 * n0 * x0) - M0;
  const int b1 = (int)floorf(2 * n1 * y0) - M1;
  float k0[2 * M0 + 1], k1[2 * M1 + 1];
#pragma unroll
  for (int t = 0; t < 2 * M0 + 1; t++) {
    const float w0 = ex[b0 + t + n0 + M0 + EPAD] - x0;
    k0[t] = __expf(geo.c0 * (w0 * w0));
  }
#pragma unroll
  for (int t = 0; t < 2 * M1 + 1; t++) {
    const float w1 = ey[b1 + t + n1 + M1 + EPAD] - y0;
    k1[t] = __expf(geo.c1 * (w1 * w1));
  }
  const float2 *gz = grid + (size_t)ty * (2 * n0) * (2 * n1);
  float sr = 0.f, si = 0.f;
#pragma unroll
  for (int t1 = 0; t1 < 2 * M1 + 1; t1++) {
    int iy = n1 + b1 + t1;                 // periodic cell of fdee2d row n1 + m1 + ell1
    const int sy = sgn_idx(iy + M1);
    iy = (iy % (2 * n1) + 2 * n1) % (2 * n1);
#pragma unroll
    for (int t0 = 0; t0 < 2 * M0 + 1; t0++) {
      int ix = n0 + b0 + t0;
      const float s = (float)(sy * sgn_idx(ix + M0));
      ix = (ix % (2 * n0) + 2 * n0) % (2 * n0);
      const float2 v = gz[(size_t)iy * (2 * n0) + ix];
      const float w = k0[t0] * k1[t1] * geo.wscale * s;
      sr += w * v.x;
      si += w * v.y;
    }
  }
  // gather2d's storage: the upper half of the detector frequencies (tx > detw/2)
  // goes, mirrored, to angle planes ntheta.. (cfunc_usfft2d packing)
  int txs = tx, tys = ty, tzs = tz;
  if (tx > detw / 2) {
    txs = detw - tx;
    tys = deth - ty - 1;
    tzs = tz + geo.ntheta;
  }
  g[(size_t)txs + (size_t)tys * (detw / 2 + 1) + (size_t)tzs * (detw / 2 + 1) * deth] =
      make_float2(sr, si);
}

// cfunc_usfft1d::fwd (cfunc_usfft1d.cu:50-66): divker1d(direction 0) with the
// fftshift sign into the periodic [2n2][n1][n0] grid (cells outside the n2
// centred rows zero), a forward FFT along the 2n2 axis, then each height
// sample gathers its 2m+1 cells (gather1d direction 0).
__global__ void u1f_load(float2 *__restrict__ grid, const float *__restrict__ f, U1Geom geo) {
  const int n0 = geo.n0, n1 = geo.n1, n2 = geo.n2;
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y;
  const int iz = blockIdx.z;  // 0 .. 2 n2 - 1
  if (tx >= n0) return;
  const int tz = iz - n2 / 2;
  float v = 0.f;
  if (tz >= 0 && tz < n2) {
    const float ker = __expf(-geo.mu2 * (tz - n2 / 2) * (tz - n2 / 2));
    v = f[(size_t)tx + (size_t)tz * n0 + (size_t)ty * n0 * n2] / ker / (2 * n2) *
        (float)sgn_idx(iz + geo.m2);
  }
  grid[(size_t)tx + (size_t)ty * n0 + (size_t)iz * n0 * n1] = make_float2(v, 0.f);
}

// Rows t of g [n1][deth/2+1][n0] for t <= deth/2, each from its own height
// z(t).  (The reference launches all deth rows and lets row deth - t write
// its value into row t as well, unconjugated: a race whose winner decides
// whether rows 0 < t < deth/2 hold g or conj(g); for real f the two differ
// only in the sign of the imaginary part.  Here every row is written once.)
__global__ void u1f_gather(float2 *__restrict__ g, const float2 *__restrict__ grid,
                           const float *__restrict__ zt, const float *__restrict__ ez,
                           U1Geom geo) {
  const int n0 = geo.n0, n1 = geo.n1, n2 = geo.n2, M = geo.m2, deth = geo.deth;
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y;
  const int t = blockIdx.z;  // 0 .. deth/2
  if (tx >= n0) return;
  const float z0 = zt[t];
  const int e0 = (int)floorf(2 * n2 * z0) - M;
  float sr = 0.f, si = 0.f;
  for (int i2 = 0; i2 < 2 * M + 1; i2++) {
    const int ell = e0 + i2;
    const float w2 = ez[ell + n2 + M + EPAD] - z0;
    const float w = geo.wscale * __expf(geo.c2 * (w2 * w2));
    int iz = n2 + ell;
    const float s = (float)sgn_idx(iz + M);
    iz = (iz % (2 * n2) + 2 * n2) % (2 * n2);
    const float2 v = grid[(size_t)tx + (size_t)ty * n0 + (size_t)iz * n0 * n1];
    sr += w * (v.x * s);
    si += w * (v.y * s);
  }
  g[(size_t)tx + (size_t)t * n0 + (size_t)ty * n0 * (deth / 2 + 1)] = make_float2(sr, si);
}

}  // namespace lam
}  // namespace tcb

using namespace tcb;
using namespace tcb::lam;

// ====================================================================== fft2d
struct tcb_fft2d {
  size_t ntheta, detw, deth;
  cufftHandle plan = 0;
};

extern "C" int tcb_fft2d_create(tcb_fft2d **out, size_t ntheta, size_t detw, size_t deth) {
  TCB_CHECK_ARG(out, "tcb_fft2d_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(ntheta >= 1 && detw >= 2 && deth >= 2 && detw % 2 == 0,
                "tcb_fft2d_create: bad sizes");
  TCB_CHECK_ARG(ntheta * deth * detw < (1ull << 40), "tcb_fft2d_create: too large");
  tcb_fft2d *h = new tcb_fft2d();
  h->ntheta = ntheta;
  h->detw = detw;
  h->deth = deth;
  int dims[2] = {(int)deth, (int)detw};
  cufftResult r = cufftPlanMany(&h->plan, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C,
                                (int)ntheta);
  if (r != CUFFT_SUCCESS) {
    delete h;
    set_error("tcb_fft2d_create: cufftPlanMany failed: %d", (int)r);
    return r == CUFFT_ALLOC_FAILED ? TCB_ERR_OUT_OF_MEMORY : TCB_ERR_CUFFT;
  }
  *out = h;
  return TCB_OK;
}

// cfunc_fft2d::fwd: g complex [ntheta][deth][detw/2+1] from f real
// [ntheta][deth][detw] (f receives the (-1)^(x+y) sign, as in the reference).
extern "C" int tcb_fft2d_fwd(tcb_fft2d *h, void *g, void *f, void *stream) {
  TCB_CHECK_ARG(h && h->plan, "tcb_fft2d_fwd: null or freed handle");
  TCB_CHECK_ARG(g && f, "tcb_fft2d_fwd: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  size_t tr = h->ntheta * h->deth * h->detw;
  size_t tc = h->ntheta * h->deth * (h->detw / 2 + 1);
  {
    StageTimer st("fft2d_sign", s);
    checker_real<<<ceil_div(tr, 256), 256, 0, s>>>((float *)f, (int)h->detw, (int)h->deth, tr);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  TCB_CUFFT(cufftSetStream(h->plan, s));
  {
    StageTimer st("fft2d_r2c", s);
    TCB_CUFFT(cufftExecR2C(h->plan, (cufftReal *)f, (cufftComplex *)g));
  }
  {
    StageTimer st("fft2d_post", s);
    fft2d_post<<<ceil_div(tc, 256), 256, 0, s>>>((float2 *)g, (int)(h->detw / 2 + 1),
                                                 (int)h->deth, tc,
                                                 1.f / (h->deth * h->detw));
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

extern "C" int tcb_fft2d_destroy(tcb_fft2d *h) {
  if (!h) return TCB_OK;
  if (h->plan) cufftDestroy(h->plan);
  delete h;
  return TCB_OK;
}

// ====================================================================== usfft2d
struct tcb_usfft2d {
  U2Geom geo;
  size_t n2;  // slabs per call
  float2 *grid = nullptr;
  float2 *cs = nullptr;
  float *ex = nullptr, *ey = nullptr;
  cufftHandle plan = 0;
  int storage = TCB_FLOAT32;  // of the stage-1 input and the output
  const float *in_scale = nullptr;  // fp16 storage scales (caller's device arrays)
  float *out_inv = nullptr;
  unsigned *maxbits = nullptr;
};

static void u2_release(tcb_usfft2d *h) {
  if (h->plan) cufftDestroy(h->plan);
  cudaFree(h->grid);
  cudaFree(h->cs);
  cudaFree(h->ex);
  cudaFree(h->ey);
  cudaFree(h->maxbits);
  h->plan = 0;
  h->grid = h->cs = nullptr;
  h->ex = h->ey = nullptr;
  h->maxbits = nullptr;
}

extern "C" int tcb_usfft2d_create(tcb_usfft2d **out, size_t n0_, size_t n1_, size_t n2_,
                                  size_t ntheta, size_t detw, size_t deth) {
  TCB_CHECK_ARG(out, "tcb_usfft2d_create: null out");
  *out = nullptr;
  // argument order of cfunc_usfft2d: (n0, n1, n2) from Python = (slabs, y, x)
  size_t n0 = n2_, n1 = n1_, n2 = n0_;
  TCB_CHECK_ARG(n0 >= (size_t)T && n1 >= (size_t)T && n0 % 2 == 0 && n1 % 2 == 0,
                "tcb_usfft2d_create: grid sizes must be even and >= %d", T);
  TCB_CHECK_ARG(n2 >= 1 && ntheta >= 1 && ntheta < (1u << 20) && detw >= 2 && deth >= 1,
                "tcb_usfft2d_create: bad sizes");
  float mu0, mu1;
  int m0, m1;
  gauss_params(n0, mu0, m0);
  gauss_params(n1, mu1, m1);
  TCB_CHECK_ARG(m0 == 4 && m1 == 4, "tcb_usfft2d_create: unexpected gridding width");
  tcb_usfft2d *h = new tcb_usfft2d();
  U2Geom &g = h->geo;
  g.n0 = (int)n0;
  g.n1 = (int)n1;
  g.m0 = m0;
  g.m1 = m1;
  g.mu0 = mu0;
  g.mu1 = mu1;
  g.ntheta = (int)ntheta;
  g.detw = (int)detw;
  g.deth = (int)deth;
  g.ntx = (int)ceil_div(2 * n0, T);
  g.nty = (int)ceil_div(2 * n1, T);
  g.wscale = (float)(LAM_PI_D / sqrtf(mu0 * mu1 * ntheta));
  g.c0 = (float)(-LAM_PI_D * LAM_PI_D / mu0);
  g.c1 = (float)(-LAM_PI_D * LAM_PI_D / mu1);
  h->n2 = n2;
  auto fail = [&](int code, const char *what) {
    set_error("tcb_usfft2d_create: %s", what);
    u2_release(h);
    delete h;
    return code;
  };
  if (cudaMalloc(&h->grid, n2 * 4 * n0 * n1 * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&h->cs, (ntheta + 1) * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&h->ex, (2 * n0 + 2 * m0 + 1 + 2 * EPAD) * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->ey, (2 * n1 + 2 * m1 + 1 + 2 * EPAD) * sizeof(float)) != cudaSuccess)
    return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  int dims[2] = {(int)(2 * n1), (int)(2 * n0)};
  if (cufftPlanMany(&h->plan, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, (int)n2) !=
      CUFFT_SUCCESS)
    return fail(TCB_ERR_CUFFT, "cufftPlanMany failed");
  if (cudaFuncSetAttribute(u2_gather<4, 4, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(U2Smem)) != cudaSuccess)
    return fail(TCB_ERR_CUDA, "smem attribute failed");
  *out = h;
  return TCB_OK;
}

static int u2_run(tcb_usfft2d *h, void *f, const void *g, const float *theta, float phi,
                  int k, int deth0, int fused, int row0, int deth_full, int nslab, int fslabs,
                  int fslab0, cudaStream_t s) {
  U2Geom geo = h->geo;
  geo.in_scale = h->storage == TCB_FLOAT16 ? h->in_scale : nullptr;
  geo.k = k;
  geo.deth0 = deth0;
  geo.fused = fused;
  geo.row0 = row0;
  geo.deth_full = deth_full;
  int tab = (int)std::max<size_t>(h->geo.ntheta,
                                  2 * std::max(geo.n0, geo.n1) + 2 * 4 + 1 + 2 * EPAD);
  u2_tables<<<ceil_div(tab, 256), 256, 0, s>>>(h->cs, h->ex, h->ey, theta, phi, geo.ntheta,
                                              geo.n0, geo.m0, geo.n1, geo.m1);
  TCB_LAUNCH_CHECK();
  count_launch();
  {
    StageTimer st("usfft2d_gather", s);
    unsigned blocks = (unsigned)(geo.ntx * geo.nty * nslab);
    if (h->storage == TCB_FLOAT16)
      u2_gather<4, 4, __half2><<<blocks, NT, sizeof(U2Smem), s>>>((const __half2 *)g, h->grid,
                                                                 h->cs, h->ex, h->ey, geo);
    else
      u2_gather<4, 4, float2><<<blocks, NT, sizeof(U2Smem), s>>>((const float2 *)g, h->grid,
                                                                h->cs, h->ex, h->ey, geo);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  TCB_CUFFT(cufftSetStream(h->plan, s));
  {
    StageTimer st("usfft2d_fft", s);
    TCB_CUFFT(cufftExecC2C(h->plan, (cufftComplex *)h->grid, (cufftComplex *)h->grid,
                           CUFFT_INVERSE));
  }
  {
    StageTimer st("usfft2d_deapod", s);
    dim3 blk(32, 8), grd(ceil_div(geo.n0, 32), ceil_div(geo.n1, 8), (unsigned)nslab);
    if (h->storage == TCB_FLOAT16) {
      const unsigned *mb = nullptr;
      if (h->out_inv) {
        const size_t gtot = (size_t)nslab * (2 * geo.n0) * (2 * geo.n1);
        TCB_CUDA(cudaMemsetAsync(h->maxbits, 0, sizeof(unsigned), s));
        absmax_c<<<std::min<unsigned>(ceil_div(gtot, 256), 148u * 16u), 256, 0, s>>>(
            h->grid, gtot, h->maxbits);
        count_launch();
        mb = h->maxbits;
      }
      u2_deapod<__half2><<<grd, blk, 0, s>>>(h->grid, (__half2 *)f, geo, nslab, fslabs, fslab0,
                                             mb, h->out_inv);
    } else {
      u2_deapod<float2><<<grd, blk, 0, s>>>(h->grid, (float2 *)f, geo, nslab, fslabs, fslab0,
                                            nullptr, nullptr);
    }
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

// cfunc_usfft2d::adj: f complex [n1][n2][n0] from g complex
// [2*ntheta][deth][detw/2+1] (packed as in usfft2d_chunks), chunk index k.
extern "C" int tcb_usfft2d_adj(tcb_usfft2d *h, void *f, const void *g, const float *theta,
                               float phi, int k, int deth0, void *stream) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft2d_adj: null or freed handle");
  TCB_CHECK_ARG(f && g && theta, "tcb_usfft2d_adj: null pointer");
  TCB_CHECK_ARG((size_t)h->geo.deth == h->n2, "tcb_usfft2d_adj: deth must equal n2 slabs");
  return u2_run(h, f, g, theta, phi, k, deth0, 0, 0, 0,
                (int)h->n2, (int)h->n2, 0, (cudaStream_t)stream);
}

// Fused form used by the device-resident chain: rows [row0, row0+nrows) of the
// full stage-1 spectrum S1 [ntheta][deth_full][detw/2+1] are gridded and the
// result is written to S2 [n1][deth_full/2+1][n0] at slabs row0.. (no packing).
extern "C" int tcb_usfft2d_adj_rows(tcb_usfft2d *h, void *S2, const void *S1,
                                    const float *theta, float phi, int row0, int nrows,
                                    int deth_full, void *stream) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft2d_adj_rows: null or freed handle");
  TCB_CHECK_ARG(S2 && S1 && theta, "tcb_usfft2d_adj_rows: null pointer");
  TCB_CHECK_ARG(nrows >= 1 && (size_t)nrows <= h->n2, "tcb_usfft2d_adj_rows: nrows > slabs");
  TCB_CHECK_ARG(row0 >= 0 && row0 + nrows <= deth_full / 2 + 1,
                "tcb_usfft2d_adj_rows: rows out of range");
  // kv of slab ty is (ty + k*deth - deth0/2)/deth0 with deth = slabs per chunk;
  // express row0 as k*deth via a geometry with deth = 1.
  tcb_usfft2d tmp = *h;
  tmp.geo.deth = 1;
  int st = u2_run(&tmp, S2, S1, theta, phi, row0, deth_full, 1, row0,
                  deth_full, nrows, deth_full / 2 + 1, row0, (cudaStream_t)stream);
  return st;
}

// cfunc_usfft2d::fwd: g complex [2*ntheta][deth][detw/2+1] (the packed layout
// that adj reads) from f complex [n1][n2][n0], chunk index k.
extern "C" int tcb_usfft2d_fwd(tcb_usfft2d *h, void *g, const void *f, const float *theta,
                               float phi, int k, int deth0, void *stream) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft2d_fwd: null or freed handle");
  TCB_CHECK_ARG(g && f && theta, "tcb_usfft2d_fwd: null pointer");
  TCB_CHECK_ARG((size_t)h->geo.deth == h->n2, "tcb_usfft2d_fwd: deth must equal n2 slabs");
  TCB_CHECK_ARG(h->geo.ntheta <= 65535 && h->geo.deth <= 65535 && 2 * h->geo.n1 <= 65535,
                "tcb_usfft2d_fwd: grid too large");
  cudaStream_t s = (cudaStream_t)stream;
  U2Geom geo = h->geo;
  geo.k = k;
  geo.deth0 = deth0;
  geo.fused = 0;
  geo.in_scale = nullptr;
  const int nslab = (int)h->n2;
  int tab = (int)std::max<size_t>(h->geo.ntheta,
                                  2 * std::max(geo.n0, geo.n1) + 2 * 4 + 1 + 2 * EPAD);
  u2_tables<<<ceil_div(tab, 256), 256, 0, s>>>(h->cs, h->ex, h->ey, theta, phi, geo.ntheta,
                                              geo.n0, geo.m0, geo.n1, geo.m1);
  TCB_LAUNCH_CHECK();
  {
    StageTimer st("usfft2d_fwd_load", s);
    u2f_load<<<dim3(ceil_div(2 * geo.n0, 256), 2 * geo.n1, nslab), 256, 0, s>>>(
        h->grid, (const float2 *)f, geo, nslab);
    TCB_LAUNCH_CHECK();
  }
  TCB_CUFFT(cufftSetStream(h->plan, s));
  {
    StageTimer st("usfft2d_fwd_fft", s);
    TCB_CUFFT(cufftExecC2C(h->plan, (cufftComplex *)h->grid, (cufftComplex *)h->grid,
                           CUFFT_FORWARD));
  }
  {
    StageTimer st("usfft2d_fwd_gather", s);
    u2f_gather<4, 4><<<dim3(ceil_div(geo.detw, 128), geo.deth, geo.ntheta), 128, 0, s>>>(
        (float2 *)g, h->grid, h->cs, h->ex, h->ey, geo);
    TCB_LAUNCH_CHECK();
  }
  count_launch(3);
  return TCB_OK;
}

// The sample positions that the gridding above uses, one per (angle, detector
// row of the call, detector column), written in take_x's layout.
__global__ void u2_positions(float *__restrict__ x, float *__restrict__ y,
                             const float2 *__restrict__ cs, U2Geom geo) {
  const size_t total = (size_t)geo.detw * geo.deth * geo.ntheta;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int tx = (int)(i % geo.detw);
  const int ty = (int)((i / geo.detw) % geo.deth);
  const int tz = (int)(i / ((size_t)geo.detw * geo.deth));
  float xv, yv;
  u2_pos(geo, cs[geo.ntheta].x, cs[tz], tx, ty, xv, yv);
  x[i] = xv;
  y[i] = yv;
}

extern "C" int tcb_usfft2d_sample_positions(tcb_usfft2d *h, float *x, float *y,
                                            const float *theta, float phi, int k, int deth0,
                                            void *stream) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft2d_sample_positions: null or freed handle");
  TCB_CHECK_ARG(x && y && theta, "tcb_usfft2d_sample_positions: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  U2Geom geo = h->geo;
  geo.k = k;
  geo.deth0 = deth0;
  int tab = (int)std::max<size_t>(h->geo.ntheta,
                                  2 * std::max(geo.n0, geo.n1) + 2 * 4 + 1 + 2 * EPAD);
  u2_tables<<<ceil_div(tab, 256), 256, 0, s>>>(h->cs, h->ex, h->ey, theta, phi, geo.ntheta,
                                              geo.n0, geo.m0, geo.n1, geo.m1);
  TCB_LAUNCH_CHECK();
  count_launch();
  const size_t total = (size_t)geo.detw * geo.deth * geo.ntheta;
  u2_positions<<<ceil_div(total, 256), 256, 0, s>>>(x, y, h->cs, geo);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

extern "C" int tcb_usfft2d_set_storage(tcb_usfft2d *h, int precision, const float *in_scale,
                                       float *out_inv_scale) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft2d_set_storage: null or freed handle");
  TCB_CHECK_ARG(precision == TCB_FLOAT32 || precision == TCB_FLOAT16,
                "tcb_usfft2d_set_storage: unknown precision %d", precision);
  h->in_scale = in_scale;
  h->out_inv = out_inv_scale;
  if (out_inv_scale && !h->maxbits && cudaMalloc(&h->maxbits, sizeof(unsigned)) != cudaSuccess) {
    cudaGetLastError();
    set_error("tcb_usfft2d_set_storage: out of device memory");
    return TCB_ERR_OUT_OF_MEMORY;
  }
  if (precision == TCB_FLOAT16)
    TCB_CUDA(cudaFuncSetAttribute(u2_gather<4, 4, __half2>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(U2Smem)));
  h->storage = precision;
  return TCB_OK;
}

extern "C" int tcb_usfft2d_destroy(tcb_usfft2d *h) {
  if (!h) return TCB_OK;
  u2_release(h);
  delete h;
  return TCB_OK;
}

// ====================================================================== usfft1d
struct tcb_usfft1d {
  U1Geom geo;
  int storage = TCB_FLOAT32;  // of the input g
  float2 *grid = nullptr;
  float *zt = nullptr, *ez = nullptr;
  cufftHandle plan = 0;
};

static void u1_release(tcb_usfft1d *h) {
  if (h->plan) cufftDestroy(h->plan);
  cudaFree(h->grid);
  cudaFree(h->zt);
  cudaFree(h->ez);
  h->plan = 0;
  h->grid = nullptr;
  h->zt = h->ez = nullptr;
}

extern "C" int tcb_usfft1d_create(tcb_usfft1d **out, size_t n0_, size_t n1_, size_t n2_,
                                  size_t deth) {
  TCB_CHECK_ARG(out, "tcb_usfft1d_create: null out");
  *out = nullptr;
  size_t n0 = n2_, n1 = n1_, n2 = n0_;  // reordered like the reference constructor
  TCB_CHECK_ARG(n0 >= 1 && n1 >= 1 && n2 >= 2 && n2 % 2 == 0 && deth >= 2,
                "tcb_usfft1d_create: bad sizes");
  TCB_CHECK_ARG(n1 < 65536 && n2 < 32768, "tcb_usfft1d_create: sizes too large");
  float mu2;
  int m2;
  gauss_params(n2, mu2, m2);
  tcb_usfft1d *h = new tcb_usfft1d();
  U1Geom &g = h->geo;
  g.n0 = (int)n0;
  g.n1 = (int)n1;
  g.n2 = (int)n2;
  g.m2 = m2;
  g.deth = (int)deth;
  g.mu2 = mu2;
  g.wscale = sqrtf((float)(LAM_PI_D / (mu2 * n0)));
  g.c2 = (float)(-LAM_PI_D * LAM_PI_D / mu2);
  auto fail = [&](int code, const char *what) {
    set_error("tcb_usfft1d_create: %s", what);
    u1_release(h);
    delete h;
    return code;
  };
  if (cudaMalloc(&h->grid, 2 * n2 * n1 * n0 * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&h->zt, deth * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->ez, (2 * n2 + 2 * m2 + 1 + 2 * EPAD) * sizeof(float)) != cudaSuccess)
    return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  int len[1] = {(int)(2 * n2)};
  int emb[1] = {(int)(n1 * n0)};
  if (cufftPlanMany(&h->plan, 1, len, emb, (int)(n1 * n0), 1, emb, (int)(n1 * n0), 1, CUFFT_C2C,
                    (int)(n0 * n1)) != CUFFT_SUCCESS)
    return fail(TCB_ERR_CUFFT, "cufftPlanMany failed");
  *out = h;
  return TCB_OK;
}

// cfunc_usfft1d::adj: f real [n1][n2][n0] from g complex [n1][deth/2+1][n0].
extern "C" int tcb_usfft1d_adj(tcb_usfft1d *h, void *f, const void *g, float phi, void *stream) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft1d_adj: null or freed handle");
  TCB_CHECK_ARG(f && g, "tcb_usfft1d_adj: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  const U1Geom &geo = h->geo;
  int tab = std::max(geo.deth, 2 * geo.n2 + 2 * geo.m2 + 1 + 2 * EPAD);
  u1_tables<<<ceil_div(tab, 256), 256, 0, s>>>(h->zt, h->ez, phi, geo.deth, geo.n2, geo.m2);
  TCB_LAUNCH_CHECK();
  count_launch();
  // z(t) = (t - deth/2)/deth * sin(phi): slope and offset for the sample search
  float sphi = sinf(phi);
  float zslope = sphi / geo.deth, zoff = -(geo.deth / 2.0f) / geo.deth * sphi;
  {
    StageTimer st("usfft1d_gather", s);
    dim3 blk(128), grd(ceil_div(geo.n0, 128), (unsigned)geo.n1, (unsigned)(2 * geo.n2));
    if (h->storage == TCB_FLOAT16)
      u1_gather<__half2><<<grd, blk, 0, s>>>((const __half2 *)g, h->grid, h->zt, h->ez, geo,
                                             zslope, zoff);
    else
      u1_gather<float2><<<grd, blk, 0, s>>>((const float2 *)g, h->grid, h->zt, h->ez, geo,
                                            zslope, zoff);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  TCB_CUFFT(cufftSetStream(h->plan, s));
  {
    StageTimer st("usfft1d_fft", s);
    TCB_CUFFT(cufftExecC2C(h->plan, (cufftComplex *)h->grid, (cufftComplex *)h->grid,
                           CUFFT_INVERSE));
  }
  {
    StageTimer st("usfft1d_deapod", s);
    dim3 blk(128), grd(ceil_div(geo.n0, 128), (unsigned)geo.n1, (unsigned)geo.n2);
    u1_deapod<<<grd, blk, 0, s>>>(h->grid, (float *)f, geo);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

// cfunc_usfft1d::fwd: g complex [n1][deth/2+1][n0] from f real [n1][n2][n0].
extern "C" int tcb_usfft1d_fwd(tcb_usfft1d *h, void *g, const void *f, float phi,
                               void *stream) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft1d_fwd: null or freed handle");
  TCB_CHECK_ARG(f && g, "tcb_usfft1d_fwd: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  const U1Geom &geo = h->geo;
  TCB_CHECK_ARG(geo.deth / 2 + 1 <= 65535, "tcb_usfft1d_fwd: deth too large");
  int tab = std::max(geo.deth, 2 * geo.n2 + 2 * geo.m2 + 1 + 2 * EPAD);
  u1_tables<<<ceil_div(tab, 256), 256, 0, s>>>(h->zt, h->ez, phi, geo.deth, geo.n2, geo.m2);
  TCB_LAUNCH_CHECK();
  {
    StageTimer st("usfft1d_fwd_load", s);
    u1f_load<<<dim3(ceil_div(geo.n0, 128), geo.n1, 2 * geo.n2), 128, 0, s>>>(
        h->grid, (const float *)f, geo);
    TCB_LAUNCH_CHECK();
  }
  TCB_CUFFT(cufftSetStream(h->plan, s));
  {
    StageTimer st("usfft1d_fwd_fft", s);
    TCB_CUFFT(cufftExecC2C(h->plan, (cufftComplex *)h->grid, (cufftComplex *)h->grid,
                           CUFFT_FORWARD));
  }
  {
    StageTimer st("usfft1d_fwd_gather", s);
    u1f_gather<<<dim3(ceil_div(geo.n0, 128), geo.n1, geo.deth / 2 + 1), 128, 0, s>>>(
        (float2 *)g, h->grid, h->zt, h->ez, geo);
    TCB_LAUNCH_CHECK();
  }
  count_launch(3);
  return TCB_OK;
}

extern "C" int tcb_usfft1d_set_storage(tcb_usfft1d *h, int precision, const float *in_scale) {
  TCB_CHECK_ARG(h && h->grid, "tcb_usfft1d_set_storage: null or freed handle");
  TCB_CHECK_ARG(precision == TCB_FLOAT32 || precision == TCB_FLOAT16,
                "tcb_usfft1d_set_storage: unknown precision %d", precision);
  h->storage = precision;
  h->geo.in_scale = precision == TCB_FLOAT16 ? in_scale : nullptr;
  return TCB_OK;
}

extern "C" int tcb_usfft1d_destroy(tcb_usfft1d *h) {
  if (!h) return TCB_OK;
  u1_release(h);
  delete h;
  return TCB_OK;
}
