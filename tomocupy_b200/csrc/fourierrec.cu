// Fourier-gridding (USFFT) backprojector for parallel-beam tomography.
//
// Same algorithm and constants as cfunc_fourierrec (src/cuda/cfunc_fourierrec.cu,
// src/include/kernels_fourierrec.cuh): 1D FFT of each projection, Gaussian
// gridding of the polar samples onto a 2x oversampled Cartesian grid
// (eps = 1e-3, half-width m = 4), 2D inverse FFT, deapodization, circular mask.
//
// B200 design (not a transcription of the reference kernels):
//  * ifftshiftc before/after the 1D FFT becomes an index shift by n/2 plus a
//    (-1)^k sign at read time, so g is transformed in a single cuFFT call.
//  * Gridding is output-stationary and atomic-free.  The periodic (2n)^2 grid
//    is cut into 32x16-cell tiles; each warp of a tile's CTA owns one 8x4
//    block of cells (one cell per lane) and keeps the accumulators of up to
//    16 slice pairs in registers.  The polar samples whose (2m+1)^2 footprint
//    reaches a tile, and for each 8x4 block the subset reaching it, depend on
//    the angles only; they are listed once when the object is created (theta
//    is fixed for the object's lifetime, as in the reference).  Per launch a
//    CTA stages the spectrum values of its samples (all pairs, pair-innermost)
//    in shared memory, and every lane adds w(cell, sample) * g[pair] for the
//    samples of its block: two exp per lane per sample serve all pairs.
//    There is no memset, no wrap pass (the grid is periodic by
//    construction), no global atomics, the summation order is fixed (results
//    are bit-reproducible) and the fftshift sign before the 2D FFT is
//    applied in the store.  Tiles are dispatched centre-first because the
//    polar sample density peaks at the origin.
//  * The 2D FFT runs on a dense (2n)^2 grid; the fftshift after it, divphi,
//    circ and (optionally) the real/imaginary unpacking of the slice pairs
//    are one kernel.
// Sample positions use the same intrinsics and operation order as takexy
// (kernels_fourierrec.cuh:23-36), so the footprint of every sample is the
// one the reference scatters to.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "fft_pow2.cuh"
#include "tcgen05.cuh"

#define TCB_PI_F 3.1415926535f

namespace tcb {
namespace fr {

constexpr int M = 4;            // gridding half-width for eps = 1e-3 (any n)
constexpr int TX = 32, TY = 16; // grid tile (cells)
constexpr int RX = 8, RY = 4;   // cell block owned by one warp (one cell per lane)
constexpr int NRX = TX / RX, NRY = TY / RY;
constexpr int NREG = NRX * NRY; // 16 blocks = 16 warps per tile
constexpr int NTH = NREG * 32;  // 512 threads
constexpr int SC = 256;         // samples staged per chunk
constexpr int SETUP_NT = 256;
// Margin of the ell/(2n) table: __cosf/__sinf may exceed 1 in magnitude by an
// ulp, which moves floor(2n*x0) one cell below -n.
constexpr int EPAD = 8;

struct Geom {
  int n, nproj, nz;
  int twon;        // 2n (grid edge)
  int ntx, nty;    // tiles per grid axis
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

// Sample position exactly as takexy computes it, and the footprint origin.
__device__ __forceinline__ void sample_pos(const float2 *__restrict__ cs,
                                           const float *__restrict__ rtab, int p, int i,
                                           float twonf, float &x0, float &y0, int &fx, int &fy) {
  float2 c = cs[p];
  float r = rtab[i];
  x0 = r * c.x;
  y0 = -(r * c.y);
  if (x0 >= 0.5f) x0 = 0.5f - 1e-5;
  if (y0 >= 0.5f) y0 = 0.5f - 1e-5;
  fx = (int)floorf(twonf * x0);
  fy = (int)floorf(twonf * y0);
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

template <int NT>
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

// Tile-local range [a, b] of the footprint cells (periodic grid) along one
// axis; returns false when the footprint misses the tile.
__device__ __forceinline__ bool local_range(int f, int origin, int width, int twon, int &a,
                                            int &b) {
  int s = f - M - origin;  // centred cells: footprint start relative to the tile
  s %= twon;
  if (s < 0) s += twon;
  if (s < width) {
    a = s;
    b = min(s + 2 * M, width - 1);
    return true;
  }
  if (s + 2 * M >= twon) {  // wraps around into the tile's start
    a = 0;
    b = s + 2 * M - twon;
    if (b >= width) b = width - 1;
    return true;
  }
  return false;
}

// ---- per-geometry sample lists ------------------------------------------
// pass 0: count the samples whose footprint reaches each tile;
// pass 1: write them (packed p*n+i) in angle-then-radius order.
// Tiles of TXT x TYT cells (ntx = ceil(2n / TXT) per row).
template <int TXT, int TYT>
__global__ void __launch_bounds__(SETUP_NT)
    list_tile_samples(const float2 *__restrict__ cs, const float *__restrict__ rtab, Geom geo,
                      int pass, int *__restrict__ counts, const long long *__restrict__ offs,
                      int *__restrict__ list) {
  __shared__ int warp_tot[SETUP_NT / 32];
  const int n = geo.n, twon = geo.twon, nproj = geo.nproj;
  const int tile = blockIdx.x;
  const int ntx = (twon + TXT - 1) / TXT;
  const int ix0 = (tile % ntx) * TXT, iy0 = (tile / ntx) * TYT;
  const int tw = min(TXT, twon - ix0), th = min(TYT, twon - iy0);
  const int X0 = ix0 - n, Y0 = iy0 - n;
  const float twonf = (float)(2 * n);
  int kx_lo = 1, kx_hi = -1, ky_lo = 1, ky_hi = -1;
  for (int k = -1; k <= 1; k++) {
    int lo = X0 - 2 * n * k, hi = X0 + tw - 1 - 2 * n * k;
    if (hi >= -n - M - 1 && lo <= n - 1 + M) { kx_lo = min(kx_lo, k); kx_hi = max(kx_hi, k); }
    lo = Y0 - 2 * n * k; hi = Y0 + th - 1 - 2 * n * k;
    if (hi >= -n - M - 1 && lo <= n - 1 + M) { ky_lo = min(ky_lo, k); ky_hi = max(ky_hi, k); }
  }
  long long base = pass ? offs[tile] : 0;
  int running = 0;
  for (int pc = 0; pc < nproj; pc += SETUP_NT) {
    int p = pc + threadIdx.x;
    int cnt = 0;
    int i0s[4], i1s[4], ks[4];
    int nr = 0;
    if (p < nproj) {
      float2 c = cs[p];
      for (int ky = ky_lo; ky <= ky_hi; ky++)
        for (int kx = kx_lo; kx <= kx_hi; kx++) {
          float ax = (float)(X0 - M - 2 * n * kx - 3), bx = (float)(X0 + tw - 1 + M - 2 * n * kx + 3);
          float ay = (float)(Y0 - M - 2 * n * ky - 3), by = (float)(Y0 + th - 1 + M - 2 * n * ky + 3);
          float lo0, hi0, lo1, hi1;
          u_interval(c.x, ax, bx, lo0, hi0);   // fx ~ u*cos, u = 2i - n
          u_interval(-c.y, ay, by, lo1, hi1);  // fy ~ -u*sin
          float lo = fmaxf(lo0, lo1), hi = fminf(hi0, hi1);
          if (lo > hi) continue;
          lo = fmaxf(lo, -2.f * n);
          hi = fminf(hi, 2.f * n);
          int i0 = max(0, (int)floorf((lo + n) * 0.5f) - 1);
          int i1 = min(n - 1, (int)ceilf((hi + n) * 0.5f) + 1);
          if (i1 < i0) continue;
          i0s[nr] = i0; i1s[nr] = i1; ks[nr] = (kx + 1) + 3 * (ky + 1);
          nr++;
        }
      for (int q = 0; q < nr; q++) {
        int kx = ks[q] % 3 - 1, ky = ks[q] / 3 - 1;
        for (int i = i0s[q]; i <= i1s[q]; i++) {
          float x0, y0;
          int fx, fy;
          sample_pos(cs, rtab, p, i, twonf, x0, y0, fx, fy);
          int ax = fx - M + 2 * n * kx, ay = fy - M + 2 * n * ky;
          if (ax <= X0 + tw - 1 && ax + 2 * M >= X0 && ay <= Y0 + th - 1 && ay + 2 * M >= Y0)
            cnt++;
        }
      }
    }
    int total;
    int off = block_exscan<SETUP_NT>(cnt, warp_tot, total);
    if (pass && p < nproj && cnt > 0) {
      int w = 0;
      for (int q = 0; q < nr; q++) {
        int kx = ks[q] % 3 - 1, ky = ks[q] / 3 - 1;
        for (int i = i0s[q]; i <= i1s[q]; i++) {
          float x0, y0;
          int fx, fy;
          sample_pos(cs, rtab, p, i, twonf, x0, y0, fx, fy);
          int ax = fx - M + 2 * n * kx, ay = fy - M + 2 * n * ky;
          if (ax <= X0 + tw - 1 && ax + 2 * M >= X0 && ay <= Y0 + th - 1 && ay + 2 * M >= Y0)
            list[base + running + off + (w++)] = p * n + i;
        }
      }
    }
    running += total;
  }
  if (!pass && threadIdx.x == 0) counts[tile] = running;
}

// pass 0: count, for each 8x4 block of each tile, the tile samples reaching
// it; pass 1: write their tile-local indices (ascending).
__global__ void __launch_bounds__(NTH)
    list_block_samples(const float2 *__restrict__ cs, const float *__restrict__ rtab, Geom geo,
                       const long long *__restrict__ toffs, const int *__restrict__ tlist,
                       int pass, int *__restrict__ counts, const long long *__restrict__ boffs,
                       int *__restrict__ blist) {
  __shared__ int wcnt[NREG][NTH / 32];
  __shared__ int run[NREG];
  const int n = geo.n, twon = geo.twon;
  const int tile = blockIdx.x;
  const int ix0 = (tile % geo.ntx) * TX, iy0 = (tile / geo.ntx) * TY;
  const int tw = min(TX, twon - ix0), th = min(TY, twon - iy0);
  const int X0 = ix0 - n, Y0 = iy0 - n;
  const float twonf = (float)(2 * n);
  const long long t0 = toffs[tile];
  const int S = (int)(toffs[tile + 1] - t0);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x < NREG) run[threadIdx.x] = 0;
  __syncthreads();
  for (int base = 0; base < S; base += NTH) {
    int k = base + threadIdx.x;
    unsigned mask = 0;
    if (k < S) {
      int s = tlist[t0 + k];
      int p = s / n, i = s % n;
      float x0, y0;
      int fx, fy, xa, xb, ya, yb;
      sample_pos(cs, rtab, p, i, twonf, x0, y0, fx, fy);
      if (local_range(fx, X0, tw, twon, xa, xb) && local_range(fy, Y0, th, twon, ya, yb)) {
        for (int ry = ya / RY; ry <= yb / RY; ry++)
          for (int rx = xa / RX; rx <= xb / RX; rx++) mask |= 1u << (ry * NRX + rx);
      }
    }
    unsigned ballots[NREG];
#pragma unroll
    for (int r = 0; r < NREG; r++) {
      ballots[r] = __ballot_sync(0xffffffffu, (mask >> r) & 1u);
      if (lane == 0) wcnt[r][wid] = __popc(ballots[r]);
    }
    __syncthreads();
    if (threadIdx.x < NREG) {  // exclusive offsets of each warp within this chunk
      int r = threadIdx.x, acc = run[r];
      for (int w = 0; w < NTH / 32; w++) {
        int c = wcnt[r][w];
        wcnt[r][w] = acc;
        acc += c;
      }
      run[r] = acc;
    }
    __syncthreads();
    if (pass) {
      unsigned lt = (1u << lane) - 1u;
#pragma unroll
      for (int r = 0; r < NREG; r++)
        if ((mask >> r) & 1u)
          blist[boffs[tile * NREG + r] + wcnt[r][wid] + __popc(ballots[r] & lt)] = k;
    }
    __syncthreads();
  }
  if (!pass && threadIdx.x < NREG) counts[tile * NREG + threadIdx.x] = run[threadIdx.x];
}

// ---- gridding --------------------------------------------------------------
// G: [nz, nproj, n] complex, plain forward FFT of each projection.
// grid: [nz, 2n, 2n] complex (fftshift sign included).
constexpr int KREC = 2 + 2 * (2 * M + 2);  // staged record: origin + 10 x-weights + 10 y-weights
template <int Z>
struct GridSmem {
  float4 g[Z / 2][SC];  // (g_z.x, g_z.y, g_z+1.x, g_z+1.y) of each staged sample
  // per staged sample: [0] tile-local footprint origin (lx0 | ly0 << 16),
  // [2..11] x-weights exp(c1 (ell/2n - x0)^2) for the 9 footprint columns and
  // a trailing 0, [12..21] the same along y.  A lane reads the weight of its
  // own column/row, so the exps are computed once per staged sample instead
  // of once per lane.
  int rec[SC][KREC];
};

// Footprint origin relative to the tile on a periodic axis, in [-2M, twon-2M-1].
__device__ __forceinline__ int tile_origin(int f, int origin, int twon) {
  int t = f - M - origin;
  t %= twon;
  if (t < 0) t += twon;
  if (t > twon - 2 * M - 1) t -= twon;
  return t;
}

template <int Z>
__global__ void __launch_bounds__(NTH, 2)
    grid_blocks(const float2 *__restrict__ G, float2 *__restrict__ grid,
                const float2 *__restrict__ cs, const float *__restrict__ rtab,
                const float *__restrict__ etab, const int *__restrict__ tile_order,
                const long long *__restrict__ toffs, const int *__restrict__ tlist,
                const long long *__restrict__ boffs, const int *__restrict__ blist, Geom geo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GridSmem<Z> &sm = *reinterpret_cast<GridSmem<Z> *>(smem_raw);
  const int n = geo.n, twon = geo.twon, nproj = geo.nproj;
  const int zgroups = (geo.nz + Z - 1) / Z;
  const int tile = tile_order[blockIdx.x / zgroups];
  const int z0 = (blockIdx.x % zgroups) * Z;
  const int ix0 = (tile % geo.ntx) * TX, iy0 = (tile / geo.ntx) * TY;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // this lane's cell, tile-local and global
  const int lx = (wid % NRX) * RX + (lane % RX);
  const int ly = (wid / NRX) * RY + (lane / RX);
  const int cx = ix0 + lx, cy = iy0 + ly;
  const int X0 = ix0 - n, Y0 = iy0 - n;
  const float twonf = (float)(2 * n);
  const int half = n / 2;
  float ar[Z], ai[Z];
#pragma unroll
  for (int z = 0; z < Z; z++) ar[z] = ai[z] = 0.f;

  const long long t0 = toffs[tile];
  const int S = (int)(toffs[tile + 1] - t0);
  long long bcur = boffs[tile * NREG + wid];
  const long long bend = boffs[tile * NREG + wid + 1];

  for (int c0 = 0; c0 < S; c0 += SC) {
    const int cnt = min(SC, S - c0);
    // stage footprint origins and separable weights
    for (int k = threadIdx.x; k < cnt; k += NTH) {
      int s = tlist[t0 + c0 + k];
      int p = s / n, i = s % n;
      float x0, y0;
      int fx, fy;
      sample_pos(cs, rtab, p, i, twonf, x0, y0, fx, fy);
      int *r = sm.rec[k];
      r[0] = (tile_origin(fx, X0, twon) & 0xFFFF) | (tile_origin(fy, Y0, twon) << 16);
      r[1] = 0;
#pragma unroll
      for (int d = 0; d < 2 * M + 1; d++) {
        float w0 = etab[fx - M + d + n + M + EPAD] - x0;
        float w1 = etab[fy - M + d + n + M + EPAD] - y0;
        r[2 + d] = __float_as_int(__expf(geo.coeff1 * w0 * w0));
        r[2 + 2 * M + 2 + d] = __float_as_int(__expf(geo.coeff1 * w1 * w1));
      }
      r[2 + 2 * M + 1] = 0;
      r[2 + 2 * (2 * M + 1) + 1] = 0;
    }
    // stage spectrum values of Z pairs, pair-innermost; consecutive threads
    // read consecutive samples of one pair (coalesced along the radius)
    for (int e = threadIdx.x; e < cnt * (Z / 2); e += NTH) {
      int k = e % cnt, zp = e / cnt;
      int s = tlist[t0 + c0 + k];
      int p = s / n, i = s % n;
      int ii = i + half;
      if (ii >= n) ii -= n;
      float sg = (i & 1) ? -geo.scale : geo.scale;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      int za = z0 + 2 * zp, zb = za + 1;
      if (za < geo.nz) {
        float2 a = G[((size_t)za * nproj + p) * n + ii];
        v.x = a.x * sg;
        v.y = a.y * sg;
      }
      if (zb < geo.nz) {
        float2 b = G[((size_t)zb * nproj + p) * n + ii];
        v.z = b.x * sg;
        v.w = b.y * sg;
      }
      sm.g[zp][k] = v;
    }
    __syncthreads();
    // this warp's samples within the chunk (block list is ascending)
    const int cend = c0 + cnt;
    while (bcur < bend) {
      int idx = (bcur + lane < bend) ? blist[bcur + lane] : 0x7fffffff;
      unsigned inb = __ballot_sync(0xffffffffu, idx < cend);
      int m = __popc(inb);
      for (int t = 0; t < m; t++) {
        int j = __shfl_sync(0xffffffffu, idx, t) - c0;
        const int *r = sm.rec[j];
        int o = r[0];
        // offset of this lane's cell in the footprint; outside -> the 0 weight
        unsigned dx = min((unsigned)(lx - (int)(short)(o & 0xFFFF)), (unsigned)(2 * M + 1));
        unsigned dy = min((unsigned)(ly - (o >> 16)), (unsigned)(2 * M + 1));
        float w = __int_as_float(r[2 + dx]) * __int_as_float(r[2 + 2 * M + 2 + dy]);
#pragma unroll
        for (int zp = 0; zp < Z / 2; zp++) {
          float4 v = sm.g[zp][j];
          ar[2 * zp] = fmaf(w, v.x, ar[2 * zp]);
          ai[2 * zp] = fmaf(w, v.y, ai[2 * zp]);
          ar[2 * zp + 1] = fmaf(w, v.z, ar[2 * zp + 1]);
          ai[2 * zp + 1] = fmaf(w, v.w, ai[2 * zp + 1]);
        }
      }
      bcur += m;
      if (m < 32) break;
    }
    __syncthreads();
  }
  // store with coeff0 and the pre-FFT fftshift sign of the (2n+2m)^2 buffer
  if (cx < twon && cy < twon) {
    int sx = 1 - 2 * ((cx + M + 1) % 2), sy = 1 - 2 * ((cy + M + 1) % 2);
    float sgn = (float)(sx * sy) * geo.coeff0;
#pragma unroll
    for (int z = 0; z < Z; z++)
      if (z0 + z < geo.nz)
        grid[((size_t)(z0 + z) * twon + cy) * twon + cx] = make_float2(ar[z] * sgn, ai[z] * sgn);
  }
}

// fftshift after the 2D FFT + divphi + circ (+ optional unpacking).
//   grid: [nz, 2n, 2n]; f complex [nz, n, n] (unpack == 0) or
//   f real [2nz, n, n] (unpack == 1).
// ---- gridding on the tensor cores (mixed precision) --------------------------
// For one 32 x 16 tile and up to 16 slice pairs, gridding is the product
//   D[cell, comp] = sum_s W[cell, s] * Gv[s, comp]
// with W[cell, s] = wx_s[cell.x - ox_s] * wy_s[cell.y - oy_s] (zero outside
// the sample's 9 x 9 footprint) and Gv the sample's spectrum values of 32
// pairs (re, im).  Per chunk of 64 listed samples the CTA writes W (512 x 64,
// fp16) and Gv (64 x 64: 32 pairs x (re, im) fp16, scaled by a power of two
// that puts max |G| at 2^13..2^14) into shared memory
// in the UMMA K-major 128-byte-swizzled layout, and one thread issues 4 M-groups
// x 4 K-steps of tcgen05.mma (M = 128 cells, N = 64, K = 16) accumulating in
// TMEM; while they run, the other CTA on the SM builds its chunk (one smem
// stage per CTA, two CTAs per SM).  The epilogue undoes the scale and
// stores like grid_blocks.  Weights and footprints are computed
// exactly as grid_blocks computes them, once per geometry, into records laid
// out in the order of the tile lists (tile_records).
constexpr int TCK = 64;                       // samples per chunk (one K block)
constexpr int TCZ = 32;                       // slice pairs per tensor-gridding CTA
constexpr int TCN = 2 * TCZ;                  // 32 pairs x (re, im)
constexpr int TCM = TX * TY;                  // 512 cells
constexpr int TC_A = TCM * TCK * 2;           // 64 KB
constexpr int TC_B = TCN * TCK * 2;           // 8 KB
constexpr int TC_STAGE = TC_A + TC_B;
constexpr int TC_THREADS = 512;

// Per-(tile, sample) record, computed once per geometry with exactly the
// arithmetic of grid_blocks, in the order of the tile lists:
// [0] tile-local footprint origin (lx0 | ly0 << 16), [1] index of the
// sample's spectrum value p*n + (i + n/2) % n with the odd-i sign in bit 31,
// [2..10] x-weights, [11..19] y-weights, [20..24] and [25..29] the byte
// offsets in W of footprint column dx and row dy (16 bits each, two per
// int; 0xFFFF outside the tile).  The sample sits at column k = (list
// position) % 64 of its chunk, so its cell (lx, ly) is at
// ly*4096 + (lx/8)*1024 + (lx%8)*128 + ((k/8 ^ lx) % 8)*16 + (k%8)*2: the
// UMMA K-major 128-byte-swizzled layout of a 512 x 64 fp16 operand.
// 128 bytes: eight int4.
constexpr int TC_REC = 32;
constexpr int TC_XO = 2 + 2 * (2 * M + 1);      // first int of the column offsets
constexpr int TC_YO = TC_XO + (2 * M + 2) / 2;  // first int of the row offsets
static_assert(TC_YO + (2 * M + 2) / 2 <= TC_REC, "record layout");

__global__ void tile_records(const float2 *__restrict__ cs, const float *__restrict__ rtab,
                             const float *__restrict__ etab, const long long *__restrict__ toffs,
                             const int *__restrict__ tlist, Geom geo, int *__restrict__ trec) {
  const int tile = blockIdx.x;
  const int n = geo.n, twon = geo.twon;
  const int ix0 = (tile % geo.ntx) * TX, iy0 = (tile / geo.ntx) * TY;
  const int X0 = ix0 - n, Y0 = iy0 - n;
  const long long t0 = toffs[tile];
  const int S = (int)(toffs[tile + 1] - t0);
  for (int k = threadIdx.x; k < S; k += blockDim.x) {
    const int sidx = tlist[t0 + k];
    const int p = sidx / n, i = sidx % n;
    float x0, y0;
    int fx, fy;
    sample_pos(cs, rtab, p, i, (float)(2 * n), x0, y0, fx, fy);
    int *r = trec + (t0 + k) * TC_REC;
    r[0] = (tile_origin(fx, X0, twon) & 0xFFFF) | (tile_origin(fy, Y0, twon) << 16);
    int ii = i + n / 2;
    if (ii >= n) ii -= n;
    r[1] = (p * n + ii) | ((i & 1) << 31);
#pragma unroll
    for (int d = 0; d < 2 * M + 1; d++) {
      float w0 = etab[fx - M + d + n + M + EPAD] - x0;
      float w1 = etab[fy - M + d + n + M + EPAD] - y0;
      r[2 + d] = __float_as_int(__expf(geo.coeff1 * w0 * w0));
      r[2 + 2 * M + 1 + d] = __float_as_int(__expf(geo.coeff1 * w1 * w1));
    }
    const int ox = tile_origin(fx, X0, twon), oy = tile_origin(fy, Y0, twon);
    const int kc = (k % TCK) >> 3, kcol = (k & 7) << 1;
    unsigned xo[2 * M + 2], yo[2 * M + 2];
#pragma unroll
    for (int d = 0; d < 2 * M + 2; d++) {
      const int lx = ox + d, ly = oy + d;
      xo[d] = (d < 2 * M + 1 && (unsigned)lx < (unsigned)TX)
                  ? (unsigned)((lx >> 3) * 1024 + (lx & 7) * 128 + (((kc ^ lx) & 7) << 4) + kcol)
                  : 0xFFFFu;
      yo[d] = (d < 2 * M + 1 && (unsigned)ly < (unsigned)TY) ? (unsigned)(ly * 4096) : 0xFFFFu;
    }
#pragma unroll
    for (int q = 0; q < (2 * M + 2) / 2; q++) {
      r[TC_XO + q] = (int)(xo[2 * q] | (xo[2 * q + 1] << 16));
      r[TC_YO + q] = (int)(yo[2 * q] | (yo[2 * q + 1] << 16));
    }
    r[TC_REC - 2] = r[TC_REC - 1] = 0;
  }
}

// One smem stage per CTA and two CTAs per SM (2 x 256 TMEM columns = all 512):
// one CTA builds its next chunk while the other's MMAs and loads are in flight.
// records in shared memory field-major, R[field * TC_RS + k], so that the
// lanes of a warp (consecutive k) read one field without bank conflicts
constexpr int TC_RS = TCK + 1;
constexpr int TC_SMEM = TC_STAGE + TC_REC * TC_RS * 4 + 64 + 1024;
constexpr uint32_t TC_IDESC = tc::idesc_f16_f32(128, TCN);
constexpr int TC_RV4 = TCK * TC_REC / 4;   // int4 per chunk of records (512)
constexpr int TC_VT = TCZ * (TCK / 8);     // value threads: (pair, 8-sample group) = 256

__global__ void absmax_kernel(const float2 *__restrict__ g, size_t total,
                              unsigned *__restrict__ out) {
  float m = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    float2 v = g[i];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(out, __float_as_uint(m));  // m >= 0: int order
}

__device__ __forceinline__ uint32_t pack_h2(__half a, __half b) {
  return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

// Tensor-core gridding of one tile and up to TCZ slice pairs.  Per chunk of
// TCK listed samples: the records (contiguous per tile, loaded as int4 one
// chunk ahead into registers), the spectrum values of 32 pairs (one thread
// per pair and 8-sample group, written as 16-byte rows of B), W zeroed and
// the footprint weights scattered; then one thread issues the MMAs.  The
// value indices run two chunks ahead so that the value loads of the next
// chunk need no dependent load.
__global__ void __launch_bounds__(TC_THREADS, 2)
    grid_tc(const float2 *__restrict__ G, float2 *__restrict__ grid,
            const int *__restrict__ tile_order, const long long *__restrict__ toffs,
            const int *__restrict__ trec, const unsigned *__restrict__ amax_bits, Geom geo,
            int *__restrict__ err) {
  using namespace tcb::tc;
  extern __shared__ uint8_t tsm_raw[];
  uint8_t *sm = tsm_raw + ((1024u - (smem_u32(tsm_raw) & 1023u)) & 1023u);
  uint8_t *A = sm, *B = sm + TC_A;
  int *R = reinterpret_cast<int *>(sm + TC_STAGE);   // [TC_REC][TC_RS]
  uint64_t *mma_done = reinterpret_cast<uint64_t *>(R + TC_REC * TC_RS);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mma_done + 2);
  const int n = geo.n, twon = geo.twon, nproj = geo.nproj;
  const int zgroups = (geo.nz + TCZ - 1) / TCZ;
  const int tile = tile_order[blockIdx.x / zgroups];
  const int z0 = (blockIdx.x % zgroups) * TCZ;
  const int ix0 = (tile % geo.ntx) * TX, iy0 = (tile / geo.ntx) * TY;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // power-of-two scale that puts max |G| in [2^13, 2^14)
  const float amax = __uint_as_float(*amax_bits);
  int ex = 0;
  if (amax > 0.f) frexpf(amax, &ex);
  const float gsc = ldexpf(1.f, 14 - ex), unsc = ldexpf(1.f, ex - 14);

  if (tid == 0) {
    mbar_init(&mma_done[0], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(tmem_slot, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const long long t0 = toffs[tile];
  const int S = (int)(toffs[tile + 1] - t0);
  const int nch = (S + TCK - 1) / TCK;
  const int4 *rec4 = reinterpret_cast<const int4 *>(trec + t0 * TC_REC);
  // value thread: pair vz, samples 8 vg .. 8 vg + 7 of a chunk
  const int vz = tid >> 3, vg = tid & 7;
  const bool vthread = tid < TC_VT && z0 + vz < geo.nz;
  const float2 *Gz = G + (size_t)(vthread ? z0 + vz : 0) * nproj * n;
  int4 prec = make_int4(0, 0, 0, 0);   // this thread's int4 of the next chunk's records
  int vi_next[8], vi_next2[8];         // value indices (with sign bit) one / two chunks ahead
  float2 pv[8];                        // the next chunk's values
  auto load_vidx = [&](int cc, int (&vi)[8]) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int k = cc * TCK + vg * 8 + j;
      vi[j] = (vthread && k < S) ? __ldg(trec + (t0 + k) * TC_REC + 1) : -1;
    }
  };
  auto load_vals = [&](const int (&vi)[8]) {
#pragma unroll
    for (int j = 0; j < 8; j++)
      pv[j] = vi[j] != -1 ? __ldg(Gz + (vi[j] & 0x7fffffff)) : make_float2(0.f, 0.f);
  };
  auto load_rec = [&](int cc) {  // int4 tid of chunk cc: record cc*TCK + tid/5
    prec = make_int4(0, 0, 0, 0);
    if (tid < TC_RV4 && cc * TCK + tid / (TC_REC / 4) < S)
      prec = __ldg(rec4 + (size_t)cc * TC_RV4 + tid);
  };
  if (nch > 0) {
    load_rec(0);
    load_vidx(0, vi_next);
    load_vals(vi_next);
    load_vidx(1, vi_next2);
  }
  bool ok = true;
  for (int c = 0; c < nch; c++) {
    const int cnt = min(TCK, S - c * TCK);
    // the MMAs of chunk c - 1 read A and B: wait for them (one thread polls)
    if (tid == 0 && c > 0 && !mbar_wait(&mma_done[0], (c - 1) & 1)) ok = false;
    ok = __syncthreads_and(ok);
    if (!ok) break;
    // (1) records of this chunk, (2) values as fp16 rows of B, (3) W = 0
    if (tid < TC_RV4) {
      const int rk = tid / (TC_REC / 4), f0 = (tid % (TC_REC / 4)) * 4;
      R[(f0 + 0) * TC_RS + rk] = prec.x;
      R[(f0 + 1) * TC_RS + rk] = prec.y;
      R[(f0 + 2) * TC_RS + rk] = prec.z;
      R[(f0 + 3) * TC_RS + rk] = prec.w;
    }
    if (tid < TC_VT) {
      uint32_t rows[2][4];  // [re, im][8 samples as 4 half2]
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        __half h[2][2];
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int vi = vi_next[j + q];
          float re = 0.f, im = 0.f;
          if (vi != -1) {
            const float sg = ((vi < 0) ? -geo.scale : geo.scale) * gsc;
            re = pv[j + q].x * sg;
            im = pv[j + q].y * sg;
          }
          h[q][0] = __float2half_rn(re);
          h[q][1] = __float2half_rn(im);
        }
#pragma unroll
        for (int c2 = 0; c2 < 2; c2++) rows[c2][j / 2] = pack_h2(h[0][c2], h[1][c2]);
      }
#pragma unroll
      for (int c2 = 0; c2 < 2; c2++) {
        const int row = vz * 2 + c2;
        *reinterpret_cast<uint4 *>(B + (row >> 3) * 1024 + (row & 7) * 128 +
                                   (((vg ^ row) & 7) << 4)) =
            make_uint4(rows[c2][0], rows[c2][1], rows[c2][2], rows[c2][3]);
      }
    }
    {
      const uint4 zero = make_uint4(0, 0, 0, 0);
      uint4 *a4 = reinterpret_cast<uint4 *>(A);
#pragma unroll
      for (int q = tid; q < TC_A / 16; q += TC_THREADS) a4[q] = zero;
    }
    __syncthreads();
    // the next chunk's records and values (and the value indices after it) fly
    // while this one is scattered and multiplied
    if (c + 1 < nch) {
      load_rec(c + 1);
#pragma unroll
      for (int j = 0; j < 8; j++) vi_next[j] = vi_next2[j];
      load_vals(vi_next);
      if (c + 2 < nch) load_vidx(c + 2, vi_next2);
    }
    // (4) footprint weights into W[cell][sample]; cell addresses are the
    // record's row offset + column offset.  Rows 0..2M-1: one (sample, row)
    // item per thread; row 2M: one cell per thread, so no thread does two
    // rows.
    static_assert(TCK * (2 * M) == TC_THREADS, "one (sample, row) item per thread");
    auto row_off = [&](const int *r, int dy) {
      return ((unsigned)r[(TC_YO + dy / 2) * TC_RS] >> ((dy & 1) * 16)) & 0xFFFFu;
    };
    {
      const int k = tid % TCK, dy = tid / TCK;
      const int *r = R + k;  // field f at r[f * TC_RS]
      const unsigned yo = k < cnt ? row_off(r, dy) : 0xFFFFu;
      if (yo != 0xFFFFu) {
        const float wyv = __int_as_float(r[(2 + 2 * M + 1 + dy) * TC_RS]);
        uint8_t *Ay = A + yo;
#pragma unroll
        for (int q = 0; q < (2 * M + 2) / 2; q++) {
          const unsigned xx = (unsigned)r[(TC_XO + q) * TC_RS];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int dx = 2 * q + h;
            const unsigned xo = (xx >> (16 * h)) & 0xFFFFu;
            if (dx < 2 * M + 1 && xo != 0xFFFFu) {
              const float w = __int_as_float(r[(2 + dx) * TC_RS]) * wyv;
              *reinterpret_cast<__half *>(Ay + xo) = __float2half_rn(w);
            }
          }
        }
      }
    }
    for (int e = tid; e < TCK * (2 * M + 1); e += TC_THREADS) {
      const int k = e % TCK, dx = e / TCK;
      if (k >= cnt) continue;
      const int *r = R + k;
      const unsigned yo = row_off(r, 2 * M);
      const unsigned xo =
          ((unsigned)r[(TC_XO + dx / 2) * TC_RS] >> ((dx & 1) * 16)) & 0xFFFFu;
      if (yo == 0xFFFFu || xo == 0xFFFFu) continue;
      const float w = __int_as_float(r[(2 + dx) * TC_RS]) *
                      __int_as_float(r[(2 + 2 * M + 1 + 2 * M) * TC_RS]);
      *reinterpret_cast<__half *>(A + yo + xo) = __float2half_rn(w);
    }
    fence_proxy_async_smem();
    __syncthreads();
    // (5) one thread issues the chunk's MMAs
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
#pragma unroll
      for (int g = 0; g < 4; g++)
#pragma unroll
        for (int kk = 0; kk < TCK / 16; kk++)
          mma_f16(tmem + g * TCN, sdesc(a0 + g * 16384 + kk * 32), sdesc(b0 + kk * 32),
                  TC_IDESC, (c > 0 || kk > 0) ? 1u : 0u);
      mma_commit(&mma_done[0]);
    }
  }
  if (tid == 0 && ok && nch > 0 && !mbar_wait(&mma_done[0], (nch - 1) & 1)) ok = false;
  ok = __syncthreads_and(ok);
  tc_fence_after();
  // Epilogue: warp w reads TMEM lanes 32(w%4).. of M-group w/4 (16 warps, 4 groups).
  const int q = warp & 3;
  {
    const int g = warp >> 2;
    const int m = g * 128 + q * 32 + lane;
    const int cx = ix0 + (m % TX), cy = iy0 + (m / TX);
    int sx = 1 - 2 * ((cx + M + 1) % 2), sy = 1 - 2 * ((cy + M + 1) % 2);
    const float sgn = (float)(sx * sy) * geo.coeff0 * unsc;
    for (int c0 = 0; c0 < TCN; c0 += 32) {
      float v[32];
      if (nch > 0) {
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(g * TCN + c0), v);
      } else {
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] = 0.f;
      }
      if (!ok || cx >= twon || cy >= twon) continue;
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int pz = c0 / 2 + j;
        if (z0 + pz < geo.nz)
          grid[((size_t)(z0 + pz) * twon + cy) * twon + cx] =
              make_float2(v[2 * j] * sgn, v[2 * j + 1] * sgn);
      }
    }
  }
  if (!ok && tid == 0) atomicOr(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// ---- gridding on the tensor cores with streamed weights ------------------------
// The same product D[cell, comp] = sum_s W[cell, s] V[s, comp] per grid tile,
// with every operand moved by copy engines instead of built by threads:
//  * W depends on the geometry only.  For 16 x 16-cell tiles (M = 256 cells,
//    two UMMA M-groups of 128) and chunks of 32 listed samples it is computed
//    once, with the fp32 gridding's arithmetic, scaled by 2^12 and by the
//    sample's fftshift sign, split into fp16 hi = fp16(w) and lo = fp16(w - hi),
//    and stored as the 16 KB shared-memory image of a K-major 64-byte-swizzled
//    operand (wimg_build).  A chunk's hi (and lo) image is one bulk copy.
//  * V holds the spectrum values of up to 64 slice pairs (N = 128 columns:
//    re, im per pair) of the chunk's 32 samples.  g16_split writes the
//    spectrum once per call as fp16 hi/lo rows [sample][comp] (pair-innermost,
//    power-of-two scaled so that max |G| is in [2^13, 2^14)); each sample's
//    256-byte row is gathered with cp.async into an MN-major 128-byte-swizzled
//    operand, so no thread converts or transposes a value.
//  * fp32 mode: W_hi V_hi + W_lo V_hi + W_hi V_lo (the lo x lo term, 2^-22
//    relative, is dropped) accumulated in fp32 in TMEM; mixed mode: W_hi V_hi.
// A ring of shared-memory stages (4 in fp32 mode, 8 in mixed mode): the
// copies of the next chunks fly while the tensor cores multiply the current
// one, across tile boundaries.  Waits are bounded (error flag).
constexpr int SW_TX = 16, SW_TY = 16;          // cells per tile
constexpr int SW_M = SW_TX * SW_TY;            // 256 cells = 2 M-groups
constexpr int SW_K = 32;                       // samples per chunk
constexpr int SW_WIMG = SW_M * SW_K * 2;       // 16 KB: one fp16 image
constexpr int SW_THREADS = 256;
constexpr float SW_WSCALE = 4096.f;            // W is stored times 2^12

// Byte offset of W element (cell row, sample k) in a K-major operand of
// 32-sample (64-byte) rows with the 64-byte swizzle (UMMA layout type 4):
// 8-row groups 512 bytes apart, 16-byte chunk k/8 of row r at chunk
// position (k/8) ^ ((r/2) % 4).
__device__ __forceinline__ uint32_t sw64_offset(int row, int k) {
  return (uint32_t)((row >> 3) * 512 + (row & 7) * 64 + ((((k >> 3) ^ (row >> 1)) & 3) << 4) +
                    ((k & 7) << 1));
}

// K-major, 64-byte swizzle: SBO = 512 (8 rows of 64 bytes), LBO unused.
__device__ __forceinline__ uint64_t sdesc_k64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(512 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)4 << 61;
  return d;
}

// Shared-memory byte offset of V element (sample k, comp c) in an MN-major
// 128-byte-swizzled operand of N comps and SW_K samples: MN atoms of 64
// comps SW_K * 128 bytes apart, K atoms of 8 samples 1024 bytes apart,
// 16-byte chunk (c % 64) / 8 of row k % 8 at chunk position
// ((c % 64) / 8) ^ (k % 8).
__device__ __forceinline__ uint32_t mn_sw128_offset(int k, int c) {
  return (uint32_t)((c >> 6) * (SW_K * 128) + (k >> 3) * 1024 + (k & 7) * 128 +
                    ((((c & 63) >> 3) ^ k) & 7) * 16 + (c & 7) * 2);
}

// MN-major, 128-byte swizzle: LBO = stride of MN atoms (lbo bytes), SBO =
// stride of K atoms (1024).  With a single MN atom (N = 64) lbo is 1024 too,
// so the descriptor addresses the same bytes whichever stride the MN atoms
// would take.
__device__ __forceinline__ uint64_t sdesc_mn(uint32_t saddr, uint32_t lbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)(lbo >> 4) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// One CTA per chunk: the chunk's W images (hi, and lo when wlo != null) and
// the spectrum row (with bit 31 clear) of each of its 32 samples (-1 = none).
__global__ void __launch_bounds__(SW_THREADS)
    wimg_build(const float2 *__restrict__ cs, const float *__restrict__ rtab,
               const float *__restrict__ etab, const long long *__restrict__ toffs,
               const int *__restrict__ tlist, const int2 *__restrict__ chunk_of,
               int ntx, Geom geo, uint4 *__restrict__ whi, uint4 *__restrict__ wlo,
               int *__restrict__ vidx) {
  extern __shared__ __align__(16) uint8_t wsm[];
  uint8_t *ihi = wsm, *ilo = wsm + SW_WIMG;
  __shared__ int s_org[SW_K];              // tile-local origin lx | ly << 16
  __shared__ float s_w[SW_K][2][2 * M + 1];  // x and y weights
  __shared__ float s_sg[SW_K];             // 2^12 times the fftshift sign of the sample
  const int c = blockIdx.x;
  const int2 co = chunk_of[c];             // (tile, first list position)
  const int tile = co.x, k0 = co.y;
  const int n = geo.n, twon = geo.twon;
  const int ix0 = (tile % ntx) * SW_TX, iy0 = (tile / ntx) * SW_TY;
  const int X0 = ix0 - n, Y0 = iy0 - n;
  const long long t0 = toffs[tile];
  const int S = (int)(toffs[tile + 1] - t0);
  const int nimg = wlo ? 2 : 1;
  for (int e = threadIdx.x; e < nimg * SW_WIMG / 16; e += SW_THREADS)
    reinterpret_cast<uint4 *>(wsm)[e] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x < SW_K) {
    const int k = threadIdx.x;
    int row = -1;
    if (k0 + k < S) {
      const int sidx = tlist[t0 + k0 + k];
      const int p = sidx / n, i = sidx % n;
      float x0, y0;
      int fx, fy;
      sample_pos(cs, rtab, p, i, (float)(2 * n), x0, y0, fx, fy);
      s_org[k] = (tile_origin(fx, X0, twon) & 0xFFFF) | (tile_origin(fy, Y0, twon) << 16);
      s_sg[k] = (i & 1) ? -SW_WSCALE : SW_WSCALE;
      // the weights as the fp32 gridding computes them (grid_blocks)
#pragma unroll
      for (int d = 0; d < 2 * M + 1; d++) {
        float w0 = etab[fx - M + d + n + M + EPAD] - x0;
        float w1 = etab[fy - M + d + n + M + EPAD] - y0;
        s_w[k][0][d] = __expf(geo.coeff1 * w0 * w0);
        s_w[k][1][d] = __expf(geo.coeff1 * w1 * w1);
      }
      int ii = i + n / 2;
      if (ii >= n) ii -= n;
      row = p * n + ii;
    } else {
      s_org[k] = 0x7FFF7FFF;  // outside every tile: no weights
    }
    vidx[(size_t)c * SW_K + k] = row;
  }
  __syncthreads();
  // 32 samples x 81 footprint cells: hi (and lo) of each weight in its cell's row
  for (int e = threadIdx.x; e < SW_K * (2 * M + 1) * (2 * M + 1); e += SW_THREADS) {
    const int k = e % SW_K, d = e / SW_K;
    const int dx = d % (2 * M + 1), dy = d / (2 * M + 1);
    const int o = s_org[k];
    if (o == 0x7FFF7FFF) continue;
    const int lx = (int)(short)(o & 0xFFFF) + dx, ly = (o >> 16) + dy;
    if (lx < 0 || lx >= SW_TX || ly < 0 || ly >= SW_TY) continue;
    // the product as grid_blocks forms it, then the exact power-of-two scale and sign
    const float w = (s_w[k][0][dx] * s_w[k][1][dy]) * s_sg[k];
    const __half h = __float2half_rn(w);
    const uint32_t off = sw64_offset(ly * SW_TX + lx, k);
    *reinterpret_cast<__half *>(ihi + off) = h;
    if (wlo) *reinterpret_cast<__half *>(ilo + off) = __float2half_rn(w - __half2float(h));
  }
  __syncthreads();
  uint4 *dh = whi + (size_t)c * (SW_WIMG / 16);
  for (int e = threadIdx.x; e < SW_WIMG / 16; e += SW_THREADS) {
    dh[e] = reinterpret_cast<const uint4 *>(ihi)[e];
    if (wlo) wlo[(size_t)c * (SW_WIMG / 16) + e] = reinterpret_cast<const uint4 *>(ilo)[e];
  }
}

// Spectrum rows for the streamed-weight gridding: pairs [zp0, zp0 + NN/2) of
// G [nz][rows] (complex) as fp16 rows [rows][NN] (pair-innermost re, im),
// hi = fp16(g * gsc) and (lo != null) lo = fp16(g * gsc - hi); absent pairs
// are zero.  A block moves 32 rows: coalesced reads per pair, 16-byte row
// writes.
template <int NN>
__global__ void __launch_bounds__(256)
    g16_split(const float2 *__restrict__ G, __half *__restrict__ hi, __half *__restrict__ lo,
              const unsigned *__restrict__ amax_bits, size_t rows, int nz, int zp0) {
  constexpr int ZP = NN / 2;
  __shared__ float2 t[32][ZP + 1];
  const size_t r0 = (size_t)blockIdx.x * 32;
  const float amax = __uint_as_float(*amax_bits);
  int ex = 0;
  if (amax > 0.f) frexpf(amax, &ex);
  const float gsc = ldexpf(1.f, 14 - ex);
  for (int e = threadIdx.x; e < 32 * ZP; e += 256) {
    const int rr = e % 32, z = e / 32;
    float2 v = make_float2(0.f, 0.f);
    if (r0 + rr < rows && zp0 + z < nz) v = G[(size_t)(zp0 + z) * rows + r0 + rr];
    t[rr][z] = make_float2(v.x * gsc, v.y * gsc);
  }
  __syncthreads();
  // each thread writes 8 comps (16 bytes) of one row
  for (int e = threadIdx.x; e < 32 * (NN / 8); e += 256) {
    const int rr = e / (NN / 8), q = e % (NN / 8);
    if (r0 + rr >= rows) continue;
    __half h[8], l[8];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float2 v = t[rr][q * 4 + j];
      h[2 * j] = __float2half_rn(v.x);
      h[2 * j + 1] = __float2half_rn(v.y);
      l[2 * j] = __float2half_rn(v.x - __half2float(h[2 * j]));
      l[2 * j + 1] = __float2half_rn(v.y - __half2float(h[2 * j + 1]));
    }
    const size_t o = (r0 + rr) * NN + (size_t)q * 8;
    *reinterpret_cast<uint4 *>(hi + o) = *reinterpret_cast<const uint4 *>(h);
    if (lo) *reinterpret_cast<uint4 *>(lo + o) = *reinterpret_cast<const uint4 *>(l);
  }
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
      : "memory");
}

// Warp roles of the streamed-weight gridding: 16 accumulator warps (warp w
// reads TMEM lanes 32 (w % 4) .. of M-group (w / 4) % 2, columns half w / 8),
// one producer warp (bulk copies of W, cp.async gathers of V) and one warp
// whose lane 0 issues the MMAs.
constexpr int WS_ACC_WARPS = 16;
constexpr int WS_THREADS = (WS_ACC_WARPS + 2) * 32;

template <int NN, bool SPLIT>
struct SwCfg {
  static constexpr int NST = SPLIT ? 4 : 8;                  // shared-memory stages
  // a chunk's gathers are published (fenced, then arrived on its stage's
  // mbarrier) once LAG newer chunks have been issued: the producer lanes wait
  // for their cp.async groups LAG deep instead of one chunk at a time
  static constexpr int LAG = NST / 2;
  static constexpr int WB = SPLIT ? 2 * SW_WIMG : SW_WIMG;   // W bytes per stage
  static constexpr int VB = SW_K * NN * 2;                   // one V operand
  static constexpr int STAGE = WB + (SPLIT ? 2 : 1) * VB;
  static constexpr int SMEM = NST * STAGE + 1024 + 256;
  // two TMEM buffers (partial sums in fp32 mode, whole tiles in mixed mode)
  // of two M-groups each
  static constexpr uint32_t TMEM_COLS = 4 * NN;
};

// fp32 mode: chunks per TMEM partial sum.  The tensor cores add each MMA's
// products into the fp32 accumulator without rounding to nearest, so an
// accumulator that takes thousands of updates (the tiles near the grid
// centre list ~25k samples at 2048 x 1500) drifts by ~1e-5 of its value;
// partial sums of SW_F chunks (256 samples) are added into fp32 registers
// instead, rounded to nearest, like the fp32 gridding's sums.
constexpr int SW_F = 8;

// Bounded wait by every lane of a warp; the lanes leave it together and agree
// on the outcome (so the warp stays converged for .sync.aligned operations).
__device__ __forceinline__ bool warp_wait(uint64_t *b, uint32_t parity) {
  const bool w = tc::mbar_wait(b, parity);
  return __all_sync(0xffffffffu, w);
}

__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(b)) : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Persistent and warp-specialised: CTA b takes the work items (tile, pair
// group) b, b + G, ... in raster order.  The producer warp streams the
// chunks of all its items through NST stages (W by bulk copies that complete
// on the stage's mbarrier, V rows by cp.async whose lanes arrive on it once
// their gathers have landed), prefetching the next chunk's row indices and
// the next item's chunk range one step ahead; the MMA warp multiplies each
// stage as it fills and releases it with tcgen05.commit; the accumulator
// warps drain each finished TMEM buffer (fp32 mode: a partial sum of SW_F
// chunks, added into registers; mixed mode: the whole tile) and release it,
// so the tensor cores fill one buffer while the other is read and a tile's
// grid cells are stored while the next tile streams in.  Every wait is
// bounded: a role that gives up sets the error flag and stops, the others
// then give up at their next wait, and the CTA lets its copies and MMAs in
// flight finish (bounded) before it frees TMEM.
template <int NN, bool SPLIT>
__global__ void __launch_bounds__(WS_THREADS, 1)
    grid_sw(const uint4 *__restrict__ whi, const uint4 *__restrict__ wlo,
            const int *__restrict__ vidx, const int2 *__restrict__ tile_chunks,
            const int *__restrict__ tile_order, int ntiles, int nitems,
            const __half *__restrict__ ghi, const __half *__restrict__ glo,
            const unsigned *__restrict__ amax_bits, float2 *__restrict__ grid, Geom geo,
            int ntx, size_t rows, int skip_empty, float *__restrict__ tscale,
            int *__restrict__ err) {
  using namespace tcb::tc;
  using Cfg = SwCfg<NN, SPLIT>;
  constexpr int NST = Cfg::NST;
  // fp16 grid (tscale != null): per-warp maxima of each pair over a tile, two
  // item parities x two column halves x 8 warps
  __shared__ float s_red[2][2][8][32];
  extern __shared__ uint8_t swsm_raw[];
  uint8_t *sm = swsm_raw + ((1024u - (smem_u32(swsm_raw) & 1023u)) & 1023u);
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + NST * Cfg::STAGE);
  uint64_t *empty = full + NST;
  uint64_t *pfull = empty + NST;  // TMEM buffer b holds a finished partial sum (tile)
  uint64_t *tfree = pfull + 2;    // TMEM buffer b was read by the accumulator warps
  uint64_t *tred = tfree + 2;     // fp16 grid: the 8 warps of column half h posted maxima
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tred + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = gridDim.x;

  if (tid == 0) {
    for (int i = 0; i < NST; i++) {
      mbar_init(&full[i], 33);  // lane 0's expect_tx arrival + 32 gather arrivals
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(&pfull[i], 1);
      mbar_init(&tfree[i], WS_ACC_WARPS);
      mbar_init(&tred[i], WS_ACC_WARPS / 2);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == WS_ACC_WARPS) {
    // ---------------- producer
    long long g = 0;      // chunks issued
    long long pub = 0;    // chunks whose gathers this lane has published
    int it = blockIdx.x;
    int2 cur = it < nitems ? tile_chunks[tile_order[it % ntiles]] : make_int2(0, 0);
    int tnext = it + G < nitems ? tile_order[(it + G) % ntiles] : 0;
    int row = cur.y > 0 ? __ldg(vidx + (size_t)cur.x * SW_K + lane) : -1;
    bool have_row = true;
    for (; it < nitems && ok; it += G) {
      // one item ahead: the next item's chunk range, the tile of the one after
      const int2 nxt = it + G < nitems ? tile_chunks[tnext] : make_int2(0, 0);
      const int tnext2 = it + 2 * G < nitems ? tile_order[(it + 2 * G) % ntiles] : 0;
      const int zg = it / ntiles;
      const __half *gh = ghi + (size_t)zg * rows * NN;
      const __half *gl = SPLIT ? glo + (size_t)zg * rows * NN : nullptr;
      if (cur.y > 0 && !have_row) row = __ldg(vidx + (size_t)cur.x * SW_K + lane);
      have_row = false;
      for (int c = 0; c < cur.y; c++, g++) {
        // the row index of the chunk after this one (possibly the next item's first)
        int row_next = -1;
        if (c + 1 < cur.y) {
          row_next = __ldg(vidx + (size_t)(cur.x + c + 1) * SW_K + lane);
        } else if (nxt.y > 0) {
          row_next = __ldg(vidx + (size_t)nxt.x * SW_K + lane);
          have_row = true;
        }
        const int s = (int)(g % NST);
        if (g >= NST && !warp_wait(&empty[s], (uint32_t)(((g / NST) + 1) & 1))) {
          ok = false;
          break;
        }
        const size_t chunk = (size_t)(cur.x + c);
        uint8_t *S = sm + s * Cfg::STAGE;
        if (lane == 0) {
          mbar_expect_tx(&full[s], (uint32_t)Cfg::WB);
          bulk_g2s(smem_u32(S), whi + chunk * (SW_WIMG / 16), SW_WIMG, &full[s]);
          if (SPLIT)
            bulk_g2s(smem_u32(S + SW_WIMG), wlo + chunk * (SW_WIMG / 16), SW_WIMG, &full[s]);
        }
        // the chunk's spectrum rows (zeros for absent samples): lane k holds the
        // row index of sample k; each step the warp copies LPR lanes' worth of
        // 16-byte pieces per row, whole rows side by side, so every warp
        // access reads full 128-byte lines
        const uint32_t vb = smem_u32(S + Cfg::WB);
        constexpr int LPR = NN / 8;         // lanes per row (16-byte pieces of a row)
        constexpr int RPS = 32 / LPR;       // rows per step
        const int q = lane % LPR;
#pragma unroll
        for (int k0 = 0; k0 < SW_K; k0 += RPS) {
          const int k = k0 + lane / LPR;
          const int rk = __shfl_sync(0xffffffffu, row, k);
          const size_t so = (size_t)(rk < 0 ? 0 : rk) * NN + (size_t)q * 8;
          const int nb = rk < 0 ? 0 : 16;
          const uint32_t d = mn_sw128_offset(k, q * 8);
          cp_async16(vb + d, gh + so, nb);
          if (SPLIT) cp_async16(vb + Cfg::VB + d, gl + so, nb);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        // chunk g - LAG's gathers have landed: publish them to the async proxy
        if (g + 1 - pub > Cfg::LAG) {
          asm volatile("cp.async.wait_group %0;" ::"n"(Cfg::LAG) : "memory");
          fence_proxy_async_smem();
          mbar_arrive(&full[pub % NST]);
          pub++;
        }
        row = row_next;
      }
      cur = nxt;
      tnext = tnext2;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    fence_proxy_async_smem();
    for (; pub < g; pub++) mbar_arrive(&full[pub % NST]);
    // the bulk copies of the last stages have landed before the CTA exits (bounded)
    for (long long gg = g > NST ? g - NST : 0; gg < g; gg++)
      mbar_wait(&full[gg % NST], (uint32_t)((gg / NST) & 1));
  } else if (warp == WS_ACC_WARPS + 1) {
    // ---------------- MMA issuer
    long long g = 0, gp = 0;  // chunks consumed, TMEM buffers started
    int it = blockIdx.x;
    int nch = it < nitems ? tile_chunks[tile_order[it % ntiles]].y : 0;
    int tnext = it + G < nitems ? tile_order[(it + G) % ntiles] : 0;
    for (; it < nitems && ok; it += G) {
      const int nch_next = it + G < nitems ? tile_chunks[tnext].y : 0;
      const int tnext2 = it + 2 * G < nitems ? tile_order[(it + 2 * G) % ntiles] : 0;
      for (int c = 0; c < nch; c++, g++) {
        const int s = (int)(g % NST);
        const bool pstart = SPLIT ? (c % SW_F == 0) : (c == 0);
        const bool pend = SPLIT ? (c % SW_F == SW_F - 1 || c == nch - 1) : (c == nch - 1);
        const uint32_t buf = (uint32_t)(gp & 1);
        // a new partial sum (tile) goes into a buffer the accumulators have read
        if (pstart && gp >= 2 && !warp_wait(&tfree[buf], (uint32_t)(((gp >> 1) + 1) & 1))) {
          ok = false;
          break;
        }
        if (!warp_wait(&full[s], (uint32_t)((g / NST) & 1))) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (lane == 0) {
          uint8_t *S = sm + s * Cfg::STAGE;
          const uint32_t a_hi = smem_u32(S), a_lo = a_hi + SW_WIMG;
          const uint32_t b_hi = smem_u32(S + Cfg::WB), b_lo = b_hi + Cfg::VB;
          constexpr uint32_t idesc = idesc_f16_f32(128, NN) | (1u << 16);  // B MN-major
          // MN atoms of the V operand (64 comps) are SW_K * 128 bytes apart
          constexpr uint32_t lbo = NN > 64 ? (uint32_t)(SW_K * 128) : 1024u;
#pragma unroll
          for (int gr = 0; gr < 2; gr++) {
            const uint32_t d = tmem + buf * 2 * NN + (uint32_t)(gr * NN);
            const uint32_t ag = (uint32_t)(gr * (SW_WIMG / 2));  // 128 rows of 64 bytes
#pragma unroll
            for (int kk = 0; kk < SW_K / 16; kk++) {
              const uint32_t acc0 = (!pstart || kk > 0) ? 1u : 0u;
              const uint64_t bh = sdesc_mn(b_hi + kk * 2048, lbo);
              mma_f16(d, sdesc_k64(a_hi + ag + kk * 32), bh, idesc, acc0);
              if (SPLIT) {
                mma_f16(d, sdesc_k64(a_lo + ag + kk * 32), bh, idesc, 1u);
                mma_f16(d, sdesc_k64(a_hi + ag + kk * 32), sdesc_mn(b_lo + kk * 2048, lbo),
                        idesc, 1u);
              }
            }
          }
          mma_commit(&empty[s]);
          if (pend) mma_commit(&pfull[buf]);
        }
        __syncwarp();
        if (pend) gp++;
      }
      nch = nch_next;
      tnext = tnext2;
    }
    // the last MMAs have finished before the CTA frees TMEM (bounded)
    if (g > 0) mbar_wait(&empty[(g - 1) % NST], (uint32_t)(((g - 1) / NST) & 1));
  } else {
    // ---------------- accumulator warps
    constexpr int HC = NN / 2;  // columns (re, im of NN / 4 pairs) per thread
    const int q = warp & 3, gr = (warp >> 2) & 1, hf = warp >> 3;
    const int m = gr * 128 + q * 32 + lane;
    const float amax = __uint_as_float(*amax_bits);
    int ex = 0;
    if (amax > 0.f) frexpf(amax, &ex);
    const float unsc = ldexpf(1.f, ex - 14) / SW_WSCALE;
    float acc[HC];
    long long gp = 0;
    long long rc = 0;  // fp16 grid: tiles whose maxima this half reduced
    int it = blockIdx.x;
    int tile = it < nitems ? tile_order[it % ntiles] : 0;
    for (; it < nitems && ok; it += G) {
      const int nch = tile_chunks[tile].y;
      const int tile_next = it + G < nitems ? tile_order[(it + G) % ntiles] : 0;
      const int nparts = SPLIT ? (nch + SW_F - 1) / SW_F : (nch > 0 ? 1 : 0);
#pragma unroll
      for (int j = 0; j < HC; j++) acc[j] = 0.f;
      for (int p = 0; p < nparts; p++, gp++) {
        const uint32_t buf = (uint32_t)(gp & 1);
        if (!warp_wait(&pfull[buf], (uint32_t)((gp >> 1) & 1))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) +
                              (uint32_t)(buf * 2 * NN + gr * NN + hf * HC);
#pragma unroll
        for (int cb = 0; cb < HC; cb += 16) {
          float v[16];
          tmem_ld16(base + cb, v);
#pragma unroll
          for (int i = 0; i < 16; i++) acc[cb + i] += v[i];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tfree[buf]);
      }
      if (!ok) break;
      // this thread's cell, pairs z0 + hf * HC / 2 ... (a tile no sample
      // reaches keeps the zeros the grid holds there when skip_empty is set)
      const int ix0 = (tile % ntx) * SW_TX, iy0 = (tile / ntx) * SW_TY;
      const int cx = ix0 + (m % SW_TX), cy = iy0 + (m / SW_TX);
      const bool store = !(skip_empty && nch == 0);
      const int sx = 1 - 2 * ((cx + M + 1) % 2), sy = 1 - 2 * ((cy + M + 1) % 2);
      const float sgn = (float)(sx * sy) * geo.coeff0 * (geo.scale * unsc);
      const int pz0 = (it / ntiles) * (NN / 2) + hf * (HC / 2);
      const size_t plane = (size_t)geo.twon * geo.twon;
      if (tscale != nullptr) {
        // fp16 grid (every tile lies inside the grid): each pair's values of
        // the tile scaled by a power of two that puts their maximum |value|
        // in [2^13, 2^14); the inverse scale goes to tscale[pair][tile]
        if (store) {
          const int par = (int)(rc & 1);
          float mine = 0.f;  // lane j: this warp's maximum of pair j
#pragma unroll
          for (int j = 0; j < HC / 2; j++) {
            const float a = fmaxf(fabsf(acc[2 * j]), fabsf(acc[2 * j + 1])) * fabsf(sgn);
            const unsigned r = __reduce_max_sync(0xffffffffu, __float_as_uint(a));
            if (lane == j) mine = __uint_as_float(r);
          }
          s_red[par][hf][warp & 7][lane] = mine;
          __syncwarp();
          if (lane == 0) mbar_arrive(&tred[hf]);
          if (!warp_wait(&tred[hf], (uint32_t)(rc & 1))) {
            ok = false;
            break;
          }
          float mx = 0.f;
#pragma unroll
          for (int w = 0; w < 8; w++) mx = fmaxf(mx, s_red[par][hf][w][lane]);
          int e = 0;
          if (mx > 0.f) frexpf(mx, &e);
          const float sc = mx > 0.f ? ldexpf(1.f, 14 - e) : 1.f;  // lane j: pair j
          if ((warp & 7) == 0 && lane < HC / 2 && pz0 + lane < geo.nz)
            tscale[(size_t)(pz0 + lane) * ntiles + tile] = mx > 0.f ? ldexpf(1.f, e - 14) : 0.f;
          __half2 *hp0 = reinterpret_cast<__half2 *>(grid) + ((size_t)pz0 * geo.twon + cy) * geo.twon + cx;
#pragma unroll
          for (int j = 0; j < HC / 2; j++) {
            const float f = sgn * __shfl_sync(0xffffffffu, sc, j);
            if (pz0 + j < geo.nz) hp0[j * plane] = __floats2half2_rn(acc[2 * j] * f, acc[2 * j + 1] * f);
          }
          rc++;
        }
      } else if (cx < geo.twon && cy < geo.twon && store) {
        float2 *gp0 = grid + ((size_t)pz0 * geo.twon + cy) * geo.twon + cx;
#pragma unroll
        for (int j = 0; j < HC / 2; j++)
          if (pz0 + j < geo.nz) gp0[j * plane] = make_float2(acc[2 * j] * sgn, acc[2 * j + 1] * sgn);
      }
      tile = tile_next;
    }
  }
  if (!ok && lane == 0) atomicOr(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, Cfg::TMEM_COLS);
  }
}

// Deapodization of output pixel (tx, ty) from the inverse-FFT value at grid
// index (tx + n/2, ty + 1 + n/2): the post-FFT fftshift sign, divphi
// (exp(mu n^2 (dx^2 + dy^2)) / nproj with dx = tx/n - 0.5, and the
// (1 - n%4) sign) and the circle mask 4x^2 + 4y^2 < 1 with x = (tx - n/2)/n
// (kernels_fourierrec.cuh divphi + circ).  The per-index terms are computed
// once per geometry with the same float arithmetic:
// tab[i] = {i/n - 0.5, (i - n/2)/n, sx(i), sy(i)}, the last two the fftshift
// signs of column index i and of row index i.  The per-pixel expressions
// keep their original form, so the circle test rounds (and contracts) as
// the reference's does on boundary pixels.
__global__ void deapod_terms(float4 *__restrict__ tab, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float d = i / (float)n - 0.5;
  const float q = (i - n / 2) / float(n);
  const int ix = i + n / 2, iy = i + 1 + n / 2;
  const int sx = 1 - 2 * ((ix + M + 1) % 2), sy = 1 - 2 * ((iy + M + 1) % 2);
  tab[i] = make_float4(d, q, (float)sx, (float)sy);
}

// Deapodized value from the terms of column tx (X) and row ty (Y);
// mun2 = mu * n^2, nsign = 1 - n % 4.
__device__ __forceinline__ float2 deapod_terms_value(float2 v, const float4 X, const float4 Y,
                                                     float mun2, int nproj, float nsign) {
  const float sgn = X.z * Y.w;
  v.x *= sgn;
  v.y *= sgn;
  const float dx = X.x, dy = Y.x, x = X.y, y = Y.y;
  float phi = __expf(mun2 * (dx * dx + dy * dy)) / nproj;
  phi *= nsign;
  v.x *= phi;
  v.y *= phi;
  const float lam = (float)((4 * x * x + 4 * y * y) < 1);
  v.x *= lam;
  v.y *= lam;
  return v;
}

template <typename OutT>
__device__ __forceinline__ void store_out(OutT *f, float2 v, int tx, int ty, int tz, const Geom &geo,
                                          int unpack) {
  const int n = geo.n;
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

// fftshift after the 2D FFT + divphi + circ (+ optional unpacking).
//   grid: [nz, 2n, 2n]; f complex [nz, n, n] (unpack == 0) or
//   f real [2nz, n, n] (unpack == 1).
template <typename OutT>
__global__ void deapod_kernel(const float2 *__restrict__ grid, OutT *__restrict__ f,
                              const float4 *__restrict__ dtab, Geom geo, int unpack) {
  const int n = geo.n, twon = geo.twon;
  int tx = blockIdx.x * blockDim.x + threadIdx.x;
  int ty = blockIdx.y * blockDim.y + threadIdx.y;
  int tz = blockIdx.z;
  if (tx >= n || ty >= n) return;
  int ix = tx + n / 2, iy = ty + 1 + n / 2;
  float2 v = grid[(size_t)tz * twon * twon + (size_t)iy * twon + ix];
  store_out(f,
            deapod_terms_value(v, __ldg(dtab + tx), __ldg(dtab + ty), geo.mu * (n * n),
                               geo.nproj, (float)(1 - n % 4)),
            tx, ty, tz, geo, unpack);
}

// Own pruned inverse 2D FFT for power-of-two 2n (N = 2n).
// Pass 1 (columns): CPC adjacent columns x of one pair's N x N grid per
// block; the inverse FFT along y keeps rows y' in [n/2 + 1, 3n/2 + 1), the
// only ones deapodization reads, in t1[pair][y' - n/2 - 1][x] (n x N).
template <int N>
__global__ void __launch_bounds__(1024) ifft_cols(const float2 *__restrict__ grid,
                                                 float2 *__restrict__ t1,
                                                 const float2 *__restrict__ tw, int cpc) {
  extern __shared__ float2 fsm[];
  constexpr int SSTR = fftk::Plan<N>::PADDED + 4;
  const int c = threadIdx.x % cpc, tid = threadIdx.x / cpc;
  const int ncb = N / cpc;
  const int z = blockIdx.x / ncb, x = (blockIdx.x % ncb) * cpc + c;
  const float2 *src = grid + (size_t)z * N * N + x;
  float2 *dst = t1 + (size_t)z * (N / 2) * N + x;
  auto in = [src](int e) { return __ldg(src + (size_t)e * N); };
  auto out = [dst](int o, float2 v) {
    const unsigned r = (unsigned)(o - (N / 4 + 1));
    if (r < (unsigned)(N / 2)) dst[(size_t)r * N] = v;
  };
  fftk::ifft<N>(fsm + c * SSTR, tid, tw, in, out);
}

// Pass 2 (rows): one kept row ty of t1 per block; the inverse FFT along x
// keeps x' in [n/2, 3n/2) and applies deapodization and the output layout.
template <int N, typename OutT>
__global__ void __launch_bounds__(N / 16, (16384 / N < 16 ? 16384 / N : 16)) ifft_rows_deapod(const float2 *__restrict__ t1,
                                                          OutT *__restrict__ f,
                                                          const float2 *__restrict__ tw,
                                                          const float4 *__restrict__ dtab,
                                                          Geom geo, int unpack) {
  extern __shared__ float2 fsm[];
  constexpr int n = N / 2;
  const int ty = blockIdx.x % n, z = blockIdx.x / n;
  const float2 *src = t1 + ((size_t)z * n + ty) * N;
  const float4 Y = __ldg(dtab + ty);
  const float mun2 = geo.mu * (n * n), nsign = (float)(1 - n % 4);
  auto in = [src](int e) { return __ldg(src + e); };
  auto out = [&](int o, float2 v) {
    const unsigned tx = (unsigned)(o - N / 4);
    if (tx < (unsigned)n)
      store_out(f, deapod_terms_value(v, __ldg(dtab + tx), Y, mun2, geo.nproj, nsign), (int)tx,
                ty, z, geo, unpack);
  };
  fftk::ifft<N>(fsm, threadIdx.x, tw, in, out);
}

// Rows-first order.  Pass 1 (rows): one row y of a pair's N x N grid per
// block; the inverse FFT along x keeps x' in [n/2, 3n/2) and writes column
// c = x' - n/2 to t1[pair][c / GW][y][c % GW].  Only n of the N outputs are
// written.  GW trades the two passes' access segments: a warp of pass 1
// stores 32 consecutive columns as 32/GW segments of 8*GW bytes; a warp of
// pass 2 (4 columns x 8 rows) loads 8 rows of 32 bytes at a row stride of
// 8*GW bytes.  2n = 4096, 2048-slice volume (rows + columns pass): GW = 16
// 35.5 + 44.5 ms, GW = 8 38.0 + 40.2 ms, GW = 4 41.0 + 38.0 ms.
constexpr int T1_GW = 8;  // default columns per group of the row-pass output (n >= 128)

template <int N, int GW = T1_GW>
__global__ void __launch_bounds__(N / 16, (16384 / N < 16 ? 16384 / N : 16))
    ifft_rows_first(const float2 *__restrict__ grid, float2 *__restrict__ t1,
                    const float2 *__restrict__ tw) {
  extern __shared__ float2 fsm[];
  constexpr int n = N / 2;
  const size_t row = blockIdx.x;  // pair * N + y
  const int y = (int)(row % N);
  const float2 *src = grid + row * N;
  float2 *dst = t1 + (row - y) * n + (size_t)y * GW;  // pair base + row offset in a group
  auto in = [src](int e) { return __ldg(src + e); };
  auto out = [&](int o, float2 v) {
    const unsigned x = (unsigned)(o - N / 4);
    if (x < (unsigned)n) dst[(size_t)(x / GW) * N * GW + x % GW] = v;
  };
  fftk::ifft<N>(fsm, threadIdx.x, tw, in, out);
}

// Pass 1 on an fp16 grid (mixed precision): cell (x, y) of pair z holds
// value / tscale[z][tile(x, y)], tiles of 16 x 16 cells; the row is scaled
// back to fp32 as it is read.
template <int N, int GW = T1_GW>
__global__ void __launch_bounds__(N / 16, (16384 / N < 16 ? 16384 / N : 16))
    ifft_rows_first_h(const __half2 *__restrict__ hgrid, const float *__restrict__ tscale,
                      float2 *__restrict__ t1, const float2 *__restrict__ tw) {
  extern __shared__ float2 fsm[];
  constexpr int n = N / 2;
  constexpr int NTX = N / 16;
  const size_t row = blockIdx.x;  // pair * N + y
  const int y = (int)(row % N);
  const size_t pair = row / N;
  const __half2 *src = hgrid + row * N;
  const float *srow = tscale + pair * (size_t)NTX * NTX + (size_t)(y / 16) * NTX;
  float2 *dst = t1 + (row - y) * n + (size_t)y * GW;
  // the row's NTX tile scales, staged once (N / 16 threads: one each)
  __shared__ float s_sc[NTX];
  s_sc[threadIdx.x] = __ldg(srow + threadIdx.x);
  __syncthreads();
  auto in = [src](int e) {
    const float2 v = __half22float2(src[e]);
    const float c = s_sc[e / 16];
    return make_float2(v.x * c, v.y * c);
  };
  auto out = [dst](int o, float2 v) {
    const unsigned x = (unsigned)(o - N / 4);
    if (x < (unsigned)n) dst[(size_t)(x / GW) * N * GW + x % GW] = v;
  };
  fftk::ifft<N>(fsm, threadIdx.x, tw, in, out);
}

// Pass 2 (columns): CPC adjacent columns tx of t1 per block; the inverse
// FFT along y keeps y' in [n/2 + 1, 3n/2 + 1) and applies deapodization and
// the output layout (ty = y' - n/2 - 1).
template <int N, typename OutT, int GW = T1_GW>
__global__ void __launch_bounds__(1024) ifft_cols_deapod(const float2 *__restrict__ t1,
                                                         OutT *__restrict__ f,
                                                         const float2 *__restrict__ tw,
                                                         const float4 *__restrict__ dtab,
                                                         Geom geo, int unpack, int cpc) {
  extern __shared__ float2 fsm[];
  constexpr int n = N / 2;
  constexpr int SSTR = fftk::Plan<N>::PADDED + 4;
  const int c = threadIdx.x % cpc, tid = threadIdx.x / cpc;
  const int ncb = n / cpc;
  const int z = blockIdx.x / ncb, tx = (blockIdx.x % ncb) * cpc + c;
  // column tx in its group of T1_GW columns (row stride T1_GW)
  const float2 *src = t1 + (size_t)z * N * n + (size_t)(tx / GW) * N * GW + tx % GW;
  const float4 X = __ldg(dtab + tx);
  const float mun2 = geo.mu * (n * n), nsign = (float)(1 - n % 4);
  auto in = [src](int e) { return __ldg(src + (size_t)e * GW); };
  auto out = [&](int o, float2 v) {
    const unsigned ty = (unsigned)(o - (N / 4 + 1));
    if (ty < (unsigned)n)
      store_out(f, deapod_terms_value(v, X, __ldg(dtab + ty), mun2, geo.nproj, nsign), tx,
                (int)ty, z, geo, unpack);
  };
  fftk::ifft<N>(fsm + c * SSTR, tid, tw, in, out);
}

inline int cols_per_block(int N) { return std::min(16384 / N, 16); }
inline size_t cols_smem(int N, int cpc) { return (size_t)cpc * (N + N / 16 + 4) * sizeof(float2); }
inline size_t rows_smem(int N) { return (size_t)(N + N / 16) * sizeof(float2); }

template <int N, int GW>
cudaError_t rows_first_attrs(int csm) {
  cudaError_t e = cudaFuncSetAttribute(ifft_rows_first<N, GW>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)rows_smem(N));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ifft_rows_first_h<N, GW>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_smem(N));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ifft_cols_deapod<N, float, GW>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ifft_cols_deapod<N, __half, GW>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
  return e;
}

// Rows pass, then columns pass with deapodization; t1 in groups of GW columns.
template <int N, int GW>
void rows_first_launch(const float2 *grid, float2 *t1, const float2 *tw, const float4 *dtab,
                       void *f, bool half, const Geom &geo, int unpack, size_t nz, int cpc,
                       const float *tscale, cudaStream_t s) {
  {
    StageTimer st("fr_ifft_rows", s);
    if (tscale)
      ifft_rows_first_h<N, GW><<<(unsigned)(N * nz), N / 16, rows_smem(N), s>>>(
          reinterpret_cast<const __half2 *>(grid), tscale, t1, tw);
    else
      ifft_rows_first<N, GW><<<(unsigned)(N * nz), N / 16, rows_smem(N), s>>>(grid, t1, tw);
    count_launch();
  }
  StageTimer st("fr_ifft_cols_deapod", s);
  const unsigned blocks = (unsigned)((N / 2 / cpc) * nz);
  const size_t sm = cols_smem(N, cpc);
  if (half)
    ifft_cols_deapod<N, __half, GW><<<blocks, cpc * (N / 16), sm, s>>>(
        t1, (__half *)f, tw, dtab, geo, unpack, cpc);
  else
    ifft_cols_deapod<N, float, GW><<<blocks, cpc * (N / 16), sm, s>>>(
        t1, (float *)f, tw, dtab, geo, unpack, cpc);
  count_launch();
}

template <int N>
cudaError_t own_fft_attrs() {
  const int csm = (int)cols_smem(N, cols_per_block(N));
  cudaError_t e = cudaFuncSetAttribute(ifft_cols<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       csm);
  if (e == cudaSuccess) e = rows_first_attrs<N, 4>(csm);
  if (e == cudaSuccess) e = rows_first_attrs<N, 8>(csm);
  if (e == cudaSuccess) e = rows_first_attrs<N, 16>(csm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ifft_rows_deapod<N, float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_smem(N));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ifft_rows_deapod<N, __half>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_smem(N));
  return e;
}

template <int N>
void own_fft_launch(const float2 *grid, float2 *t1, const float2 *tw, const float4 *dtab,
                    void *f, bool half, const Geom &geo, int unpack, size_t nz, int cpc,
                    bool rows_first, int gw, const float *tscale, cudaStream_t s) {
  if (rows_first) {
    if (gw == 4)
      rows_first_launch<N, 4>(grid, t1, tw, dtab, f, half, geo, unpack, nz, cpc, tscale, s);
    else if (gw == 16)
      rows_first_launch<N, 16>(grid, t1, tw, dtab, f, half, geo, unpack, nz, cpc, tscale, s);
    else
      rows_first_launch<N, 8>(grid, t1, tw, dtab, f, half, geo, unpack, nz, cpc, tscale, s);
    return;
  }
  {
    StageTimer st("fr_ifft_cols", s);
    ifft_cols<N><<<(unsigned)((N / cpc) * nz), cpc * (N / 16), cols_smem(N, cpc), s>>>(grid, t1,
                                                                                      tw, cpc);
    count_launch();
  }
  {
    StageTimer st("fr_ifft_rows_deapod", s);
    const unsigned blocks = (unsigned)((N / 2) * nz);
    if (half)
      ifft_rows_deapod<N, __half><<<blocks, N / 16, rows_smem(N), s>>>(t1, (__half *)f, tw,
                                                                       dtab, geo, unpack);
    else
      ifft_rows_deapod<N, float><<<blocks, N / 16, rows_smem(N), s>>>(t1, (float *)f, tw, dtab,
                                                                      geo, unpack);
    count_launch();
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
  long long *toffs = nullptr;  // [ntiles+1] offsets into tlist
  int *tlist = nullptr;        // samples per tile (p*n+i)
  long long *boffs = nullptr;  // [ntiles*16+1] offsets into blist
  int *blist = nullptr;        // tile-local sample indices per 8x4 block
  float2 *grid = nullptr;
  float2 *g32 = nullptr;  // fp32 staging of g (FLOAT16 only)
  cufftHandle plan1d = 0, plan2d = 0;
  // Pruned inverse 2D FFT: row transforms over all 2n rows, then column
  // transforms over only the n columns [n/2, 3n/2) that deapodization reads.
  cufftHandle plan_rows = 0, plan_cols = 0;
  bool pruned = false;
  // Own pruned FFT (rows pass, then columns pass fused with deapodization,
  // or the reverse) when 2n is a power of two in [256, 8192]: own_n = 2n,
  // else 0.
  int own_n = 0;
  int own_cpc = 0;  // columns per block of the own column pass
  int t1_gw = tcb::fr::T1_GW;  // columns per group of the row-pass output (4, 8 or 16)
  bool own_rows_first = true;  // rows pass first (columns pass fused with deapodization)
  int zblock = 0;  // pairs per gridding block (2/4/8/16; 0 = largest that fits nz)
  int grid_mode = 0;          // TCB_GRID_FP32 or TCB_GRID_TENSOR
  bool out_f16 = false;       // fp16 output slices (set_output) with fp32 input
  bool spectrum_in = false;   // g already holds the projection FFT (set_input_spectrum)
  unsigned *amax = nullptr;   // max |G| bits for the tensor-core gridding scale
  int *trec = nullptr;        // per-(tile, sample) records (tensor-core gridding)
  int *tc_err = nullptr;      // set by a tensor-core gridding wait that timed out
  float2 *t1 = nullptr;  // first-pass output: [nz][2n][n] rows first, [nz][n][2n] columns first
  float2 *tw = nullptr;  // per-stage twiddle table of the length-2n transforms
  float4 *dtab = nullptr;  // [n] deapodization terms (deapod_terms)
  int ntiles = 0;
  size_t list_bytes = 0;
  // streamed-weight tensor-core gridding (16 x 16 tiles, chunks of 64 samples)
  int sw_nn = 0;                   // comps per CTA (64 or 128); 0 = not built
  int sw_ntx = 0, sw_ntiles = 0, sw_zgroups = 0;
  long long sw_chunks = 0;
  int sw_nonempty = 0;     // tiles with at least one listed sample
  float *sw_tscale = nullptr;  // mixed: [pairs][tiles] inverse scales of the fp16 grid
  // the format in which the grid cells outside every sample footprint hold
  // zeros (0: not known, 1: fp32 grid, 2: fp16 grid); set once, then kept,
  // because only the gridding writes the grid when the inverse FFT is the
  // library's own
  int grid_zero_fmt = 0;
  bool sw_lo = false;              // lo images present (fp32 mode)
  long long *sw_toffs = nullptr;
  int *sw_tlist = nullptr;
  int2 *sw_tile_chunks = nullptr;  // per tile: first chunk, chunk count
  int *sw_order = nullptr;         // tiles centre-first
  uint4 *sw_whi = nullptr, *sw_wlo = nullptr;
  int *sw_vidx = nullptr;
  __half *sw_ghi = nullptr, *sw_glo = nullptr;
};

using namespace tcb;
using namespace tcb::fr;

namespace {

void fr_release(tcb_fourierrec *h) {
  if (h->plan1d) cufftDestroy(h->plan1d);
  if (h->plan2d) cufftDestroy(h->plan2d);
  if (h->plan_rows) cufftDestroy(h->plan_rows);
  if (h->plan_cols) cufftDestroy(h->plan_cols);
  cudaFree(h->cs);
  cudaFree(h->rtab);
  cudaFree(h->etab);
  cudaFree(h->tile_order);
  cudaFree(h->toffs);
  cudaFree(h->tlist);
  cudaFree(h->boffs);
  cudaFree(h->blist);
  cudaFree(h->grid);
  cudaFree(h->g32);
  cudaFree(h->t1);
  cudaFree(h->tw);
  cudaFree(h->dtab);
  h->dtab = nullptr;
  cudaFree(h->amax);
  cudaFree(h->tc_err);
  cudaFree(h->trec);
  h->trec = nullptr;
  cudaFree(h->sw_toffs);
  cudaFree(h->sw_tlist);
  cudaFree(h->sw_tile_chunks);
  cudaFree(h->sw_order);
  cudaFree(h->sw_whi);
  cudaFree(h->sw_wlo);
  cudaFree(h->sw_vidx);
  cudaFree(h->sw_ghi);
  cudaFree(h->sw_glo);
  cudaFree(h->sw_tscale);
  h->sw_tscale = nullptr;
  h->sw_toffs = nullptr;
  h->sw_tlist = nullptr;
  h->sw_tile_chunks = nullptr;
  h->sw_order = nullptr;
  h->sw_whi = h->sw_wlo = nullptr;
  h->sw_vidx = nullptr;
  h->sw_ghi = h->sw_glo = nullptr;
  h->sw_nn = 0;
  h->t1 = h->tw = nullptr;
  h->amax = nullptr;
  h->tc_err = nullptr;
  h->plan1d = h->plan2d = h->plan_rows = h->plan_cols = 0;
  h->cs = nullptr;
  h->rtab = h->etab = nullptr;
  h->tile_order = nullptr;
  h->toffs = h->boffs = nullptr;
  h->tlist = h->blist = nullptr;
  h->grid = h->g32 = nullptr;
}

template <int Z>
int launch_grid(tcb_fourierrec *h, const float2 *gc, cudaStream_t s) {
  const Geom &geo = h->geo;
  unsigned zgroups = (unsigned)((h->nz + Z - 1) / Z);
  grid_blocks<Z><<<(unsigned)h->ntiles * zgroups, NTH, sizeof(GridSmem<Z>), s>>>(
      gc, h->grid, h->cs, h->rtab, h->etab, h->tile_order, h->toffs, h->tlist, h->boffs,
      h->blist, geo);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

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
  if (h->own_n) {
  } else if (h->pruned) {
    TCB_CUFFT(cufftSetStream(h->plan_rows, s));
    TCB_CUFFT(cufftSetStream(h->plan_cols, s));
  } else {
    TCB_CUFFT(cufftSetStream(h->plan2d, s));
  }
  if (!h->spectrum_in) {
    StageTimer st("fr_fft1d", s);
    TCB_CUFFT(cufftExecC2C(h->plan1d, (cufftComplex *)gc, (cufftComplex *)gc, CUFFT_FORWARD));
  }
  bool grid_h = false;  // the gridding writes an fp16 grid with per-tile scales
  if (h->grid_mode == TCB_GRID_TENSOR_FP32 || h->grid_mode == TCB_GRID_TENSOR_STREAM) {
    const size_t gtot = h->nz * h->nproj * h->n;
    const size_t rows = h->nproj * h->n;
    const double nimg = h->sw_lo ? 2.0 : 1.0;
    // spectrum operand rows (fp16 hi, lo) of every pair group
    const double vbytes = (double)h->sw_zgroups * rows * h->sw_nn * 2.0 * nimg;
    {
      // algorithmic bytes: the spectrum read twice (maximum, split), the rows written
      StageTimer st("fr_split16", s, 2.0 * gtot * sizeof(float2) + vbytes);
      TCB_CUDA(cudaMemsetAsync(h->amax, 0, sizeof(unsigned), s));
      absmax_kernel<<<std::min<unsigned>(ceil_div(gtot, 256), 148u * 16u), 256, 0, s>>>(
          gc, gtot, h->amax);
      for (int zg = 0; zg < h->sw_zgroups; zg++) {
        const size_t off = (size_t)zg * rows * h->sw_nn;
        __half *lo = h->sw_lo ? h->sw_glo + off : nullptr;
        if (h->sw_nn == 128)
          g16_split<128><<<ceil_div(rows, 32), 256, 0, s>>>(gc, h->sw_ghi + off, lo, h->amax,
                                                            rows, (int)h->nz, zg * 64);
        else
          g16_split<64><<<ceil_div(rows, 32), 256, 0, s>>>(gc, h->sw_ghi + off, lo, h->amax,
                                                           rows, (int)h->nz, zg * 32);
      }
      TCB_LAUNCH_CHECK();
      count_launch(1 + h->sw_zgroups);
    }
    // with the library's own inverse FFT (which reads the grid, never writes
    // it) the cells no sample reaches are zeroed once and never rewritten
    const bool skip = h->own_n != 0;
    // mixed precision read by the own rows-first FFT: the grid is stored in
    // fp16, each pair of each tile scaled by its own power of two
    grid_h = !h->sw_lo && skip && h->own_rows_first && h->sw_tscale != nullptr &&
             geo.twon % SW_TX == 0;
    const int fmt = grid_h ? 2 : 1;
    if (skip && h->grid_zero_fmt != fmt) {
      TCB_CUDA(cudaMemsetAsync(h->grid, 0, h->nz * (size_t)geo.twon * geo.twon * sizeof(float2), s));
      if (grid_h)
        TCB_CUDA(cudaMemsetAsync(h->sw_tscale, 0, h->nz * (size_t)h->sw_ntiles * sizeof(float), s));
      h->grid_zero_fmt = fmt;
    }
    if (!skip) h->grid_zero_fmt = 0;
    // algorithmic bytes: every weight image and its sample rows streamed once,
    // the spectrum operand read once, the grid cells of the tiles written
    // (all tiles, or those samples reach); FLOPs: the products the tensor
    // cores form (3 per term in fp32 mode)
    const double C = (double)h->sw_chunks;
    const double gcells = skip ? (double)h->sw_nonempty * SW_M
                               : (double)geo.twon * geo.twon;
    StageTimer st("fr_gather_sw", s,
                  h->sw_zgroups * C * (SW_WIMG * nimg + SW_K * sizeof(int)) + vbytes +
                      (double)h->nz * gcells * (grid_h ? sizeof(__half2) : sizeof(float2)),
                  h->sw_zgroups * C * 2.0 * SW_M * h->sw_nn * SW_K * (h->sw_lo ? 3.0 : 1.0));
    // persistent: one CTA per SM (all of TMEM, ~193 KB of shared memory)
    const int nitems = h->sw_ntiles * h->sw_zgroups;
    const unsigned grd = (unsigned)std::min(nitems, sm_count());
#define FR_SW(NN_, SPLIT_)                                                                 \
  grid_sw<NN_, SPLIT_><<<grd, WS_THREADS, SwCfg<NN_, SPLIT_>::SMEM, s>>>(                  \
      h->sw_whi, h->sw_wlo, h->sw_vidx, h->sw_tile_chunks, h->sw_order, h->sw_ntiles,       \
      nitems, h->sw_ghi, h->sw_glo, h->amax, h->grid, geo, h->sw_ntx, rows, skip ? 1 : 0,   \
      grid_h ? h->sw_tscale : nullptr, h->tc_err)
    if (h->sw_nn == 128) {
      if (h->sw_lo) FR_SW(128, true); else FR_SW(128, false);
    } else {
      if (h->sw_lo) FR_SW(64, true); else FR_SW(64, false);
    }
#undef FR_SW
    TCB_LAUNCH_CHECK();
    count_launch();
  } else if (h->grid_mode == TCB_GRID_TENSOR) {
    StageTimer st("fr_gather_tc", s);
    const size_t gtot = h->nz * h->nproj * h->n;
    TCB_CUDA(cudaMemsetAsync(h->amax, 0, sizeof(unsigned), s));
    absmax_kernel<<<std::min<unsigned>(ceil_div(gtot, 256), 148u * 16u), 256, 0, s>>>(gc, gtot,
                                                                                      h->amax);
    const unsigned zgroups = (unsigned)((h->nz + TCZ - 1) / TCZ);
    grid_tc<<<(unsigned)h->ntiles * zgroups, TC_THREADS, TC_SMEM, s>>>(
        gc, h->grid, h->tile_order, h->toffs, h->trec, h->amax, geo, h->tc_err);
    TCB_LAUNCH_CHECK();
    count_launch(2);
    h->grid_zero_fmt = h->own_n ? 1 : 0;  // every cell written, fp32
  } else {
    StageTimer st("fr_gather", s);
    int rc;
    const size_t zb = h->zblock ? (size_t)h->zblock : 16;
    h->grid_zero_fmt = h->own_n ? 1 : 0;  // every cell written, fp32
    if (h->nz >= 16 && zb >= 16) rc = launch_grid<16>(h, gc, s);
    else if (h->nz >= 8 && zb >= 8) rc = launch_grid<8>(h, gc, s);
    else if (h->nz >= 4 && zb >= 4) rc = launch_grid<4>(h, gc, s);
    else rc = launch_grid<2>(h, gc, s);
    if (rc != TCB_OK) return rc;
  }
  const bool out_half = h->precision == TCB_FLOAT16 || h->out_f16;
  if (h->own_n) {
    const bool half = out_half;
    const int cpc = h->own_cpc;
    const bool rf = h->own_rows_first;
    const int gw = h->t1_gw;
    const float *ts = grid_h ? h->sw_tscale : nullptr;  // the gridding wrote an fp16 grid
    switch (h->own_n) {
      case 256: own_fft_launch<256>(h->grid, h->t1, h->tw, h->dtab, f, half, geo, unpack, h->nz, cpc, rf, gw, ts, s); break;
      case 512: own_fft_launch<512>(h->grid, h->t1, h->tw, h->dtab, f, half, geo, unpack, h->nz, cpc, rf, gw, ts, s); break;
      case 1024: own_fft_launch<1024>(h->grid, h->t1, h->tw, h->dtab, f, half, geo, unpack, h->nz, cpc, rf, gw, ts, s); break;
      case 2048: own_fft_launch<2048>(h->grid, h->t1, h->tw, h->dtab, f, half, geo, unpack, h->nz, cpc, rf, gw, ts, s); break;
      case 4096: own_fft_launch<4096>(h->grid, h->t1, h->tw, h->dtab, f, half, geo, unpack, h->nz, cpc, rf, gw, ts, s); break;
      default: own_fft_launch<8192>(h->grid, h->t1, h->tw, h->dtab, f, half, geo, unpack, h->nz, cpc, rf, gw, ts, s); break;
    }
    TCB_LAUNCH_CHECK();
    return TCB_OK;
  }
  {
    StageTimer st("fr_fft2d", s);
    if (h->pruned) {
      // separable: all rows along x, then the kept columns along y, per pair
      TCB_CUFFT(cufftExecC2C(h->plan_rows, (cufftComplex *)h->grid, (cufftComplex *)h->grid,
                             CUFFT_INVERSE));
      const size_t plane = (size_t)geo.twon * geo.twon;
      for (size_t z = 0; z < h->nz; z++) {
        cufftComplex *c = (cufftComplex *)(h->grid + z * plane + h->n / 2);
        TCB_CUFFT(cufftExecC2C(h->plan_cols, c, c, CUFFT_INVERSE));
      }
    } else {
      TCB_CUFFT(cufftExecC2C(h->plan2d, (cufftComplex *)h->grid, (cufftComplex *)h->grid,
                             CUFFT_INVERSE));
    }
  }
  {
    StageTimer st("fr_deapod", s);
    dim3 blk(32, 8), grd(ceil_div(h->n, 32), ceil_div(h->n, 8), (unsigned)h->nz);
    if (out_half)
      deapod_kernel<__half><<<grd, blk, 0, s>>>(h->grid, (__half *)f, h->dtab, geo, unpack);
    else
      deapod_kernel<float><<<grd, blk, 0, s>>>(h->grid, (float *)f, h->dtab, geo, unpack);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

// Exclusive prefix sums of device counts -> device offsets (setup only).
int scan_counts(const int *d_counts, long long *d_offs, size_t count, long long &total) {
  std::vector<int> c(count);
  std::vector<long long> o(count + 1);
  TCB_CUDA(cudaMemcpy(c.data(), d_counts, count * sizeof(int), cudaMemcpyDeviceToHost));
  o[0] = 0;
  for (size_t k = 0; k < count; k++) o[k + 1] = o[k] + c[k];
  TCB_CUDA(cudaMemcpy(d_offs, o.data(), (count + 1) * sizeof(long long),
                      cudaMemcpyHostToDevice));
  total = o[count];
  return TCB_OK;
}

// Build the per-tile and per-block sample lists (depends on theta and n only).
int build_lists(tcb_fourierrec *h) {
  const Geom &geo = h->geo;
  const int nt = h->ntiles;
  int *counts = nullptr;
  TCB_CUDA(cudaMalloc(&counts, (size_t)nt * NREG * sizeof(int)));
  int st = TCB_OK;
  long long ntot = 0, nbtot = 0;
  do {
    list_tile_samples<TX, TY><<<nt, SETUP_NT>>>(h->cs, h->rtab, geo, 0, counts, nullptr,
                                                nullptr);
    if (cudaGetLastError() != cudaSuccess) { st = TCB_ERR_CUDA; break; }
    if ((st = scan_counts(counts, h->toffs, nt, ntot)) != TCB_OK) break;
    if (cudaMalloc(&h->tlist, std::max<long long>(ntot, 1) * sizeof(int)) != cudaSuccess) {
      st = TCB_ERR_OUT_OF_MEMORY;
      break;
    }
    list_tile_samples<TX, TY><<<nt, SETUP_NT>>>(h->cs, h->rtab, geo, 1, nullptr, h->toffs,
                                                h->tlist);
    list_block_samples<<<nt, NTH>>>(h->cs, h->rtab, geo, h->toffs, h->tlist, 0, counts,
                                    nullptr, nullptr);
    if (cudaGetLastError() != cudaSuccess) { st = TCB_ERR_CUDA; break; }
    if ((st = scan_counts(counts, h->boffs, (size_t)nt * NREG, nbtot)) != TCB_OK) break;
    if (cudaMalloc(&h->blist, std::max<long long>(nbtot, 1) * sizeof(int)) != cudaSuccess) {
      st = TCB_ERR_OUT_OF_MEMORY;
      break;
    }
    list_block_samples<<<nt, NTH>>>(h->cs, h->rtab, geo, h->toffs, h->tlist, 1, nullptr,
                                    h->boffs, h->blist);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      set_error("fourierrec: list construction failed: %s", cudaGetErrorString(e));
      st = TCB_ERR_CUDA;
      break;
    }
  } while (0);
  cudaFree(counts);
  if (st == TCB_ERR_OUT_OF_MEMORY) set_error("fourierrec: out of memory for sample lists");
  if (st == TCB_ERR_CUDA && tcb_last_error()[0] == 0) set_error("fourierrec: list kernel failed");
  h->list_bytes = (size_t)(ntot + nbtot) * sizeof(int);
  return st;
}

// Streamed-weight gridding tables: sample lists of 16 x 16 tiles, their chunks
// of 64, the weight images (hi, and lo for fp32) and the spectrum rows of
// every chunk, tiles centre-first; and the per-call fp16 spectrum buffers.
int sw_build(tcb_fourierrec *h, bool with_lo) {
  const Geom &geo = h->geo;
  const int ntx = (geo.twon + SW_TX - 1) / SW_TX, nty = (geo.twon + SW_TY - 1) / SW_TY;
  const int nt = ntx * nty;
  const int nn = h->nz > 32 ? 128 : 64;
  const int zgroups = (int)((h->nz + nn / 2 - 1) / (nn / 2));
  const size_t rows = h->nproj * h->n;
  int *counts = nullptr;
  int2 *chunk_of = nullptr;
  auto oom = [&](const char *what) {
    cudaGetLastError();
    cudaFree(counts);
    cudaFree(chunk_of);
    set_error("tcb_fourierrec_set_gridding: out of device memory (%s)", what);
    return TCB_ERR_OUT_OF_MEMORY;
  };
  if (!h->sw_toffs) {
    if (cudaMalloc(&counts, (size_t)nt * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->sw_toffs, ((size_t)nt + 1) * sizeof(long long)) != cudaSuccess)
      return oom("tile offsets");
    list_tile_samples<SW_TX, SW_TY><<<nt, SETUP_NT>>>(h->cs, h->rtab, geo, 0, counts, nullptr,
                                                      nullptr);
    TCB_CUDA(cudaGetLastError());
    long long total = 0;
    int st = scan_counts(counts, h->sw_toffs, nt, total);
    cudaFree(counts);
    counts = nullptr;
    if (st != TCB_OK) return st;
    if (cudaMalloc(&h->sw_tlist, std::max<long long>(total, 1) * sizeof(int)) != cudaSuccess)
      return oom("tile lists");
    list_tile_samples<SW_TX, SW_TY><<<nt, SETUP_NT>>>(h->cs, h->rtab, geo, 1, nullptr,
                                                      h->sw_toffs, h->sw_tlist);
    TCB_CUDA(cudaGetLastError());
  }
  // chunks of 64 listed samples per tile
  std::vector<long long> toffs(nt + 1);
  TCB_CUDA(cudaMemcpy(toffs.data(), h->sw_toffs, (nt + 1) * sizeof(long long),
                      cudaMemcpyDeviceToHost));
  std::vector<int2> tch(nt);
  std::vector<int2> cof;
  for (int t = 0; t < nt; t++) {
    const long long S = toffs[t + 1] - toffs[t];
    const int nc = (int)((S + SW_K - 1) / SW_K);
    tch[t] = make_int2((int)cof.size(), nc);
    for (int j = 0; j < nc; j++) cof.push_back(make_int2(t, j * SW_K));
  }
  const long long C = (long long)cof.size();
  TCB_CHECK_ARG(C < (1ll << 31), "tcb_fourierrec_set_gridding: too many chunks");
  if (!h->sw_tile_chunks &&
      cudaMalloc(&h->sw_tile_chunks, (size_t)nt * sizeof(int2)) != cudaSuccess)
    return oom("chunk table");
  TCB_CUDA(cudaMemcpy(h->sw_tile_chunks, tch.data(), nt * sizeof(int2), cudaMemcpyHostToDevice));
  // tiles in raster order: the persistent CTAs take consecutive tiles at a
  // time, so the grid rows they store at once (and the weight images they
  // stream, which are laid out in tile order) are neighbours in memory
  std::vector<int> order(nt);
  for (int t = 0; t < nt; t++) order[t] = t;
  if (!h->sw_order && cudaMalloc(&h->sw_order, (size_t)nt * sizeof(int)) != cudaSuccess)
    return oom("tile order");
  TCB_CUDA(cudaMemcpy(h->sw_order, order.data(), nt * sizeof(int), cudaMemcpyHostToDevice));
  // weight images and spectrum rows
  const size_t img = (size_t)SW_WIMG;
  if (cudaMalloc(&chunk_of, std::max<long long>(C, 1) * sizeof(int2)) != cudaSuccess)
    return oom("chunk map");
  if (cudaMalloc(&h->sw_whi, std::max<long long>(C, 1) * img) != cudaSuccess ||
      (with_lo && cudaMalloc(&h->sw_wlo, std::max<long long>(C, 1) * img) != cudaSuccess))
    return oom("weight images");
  if (!h->sw_vidx &&
      cudaMalloc(&h->sw_vidx, std::max<long long>(C, 1) * SW_K * sizeof(int)) != cudaSuccess)
    return oom("spectrum rows");
  if (!h->sw_ghi) {
    const size_t gb = (size_t)zgroups * rows * nn * sizeof(__half);
    if (cudaMalloc(&h->sw_ghi, gb) != cudaSuccess) return oom("fp16 spectrum");
  }
  if (!with_lo && !h->sw_tscale &&
      cudaMalloc(&h->sw_tscale, h->nz * (size_t)nt * sizeof(float)) != cudaSuccess)
    return oom("fp16 grid scales");
  if (with_lo && !h->sw_glo) {
    const size_t gb = (size_t)zgroups * rows * nn * sizeof(__half);
    if (cudaMalloc(&h->sw_glo, gb) != cudaSuccess) return oom("fp16 spectrum");
  }
  TCB_CUDA(cudaMemcpy(chunk_of, cof.data(), C * sizeof(int2), cudaMemcpyHostToDevice));
  const int wsm = (with_lo ? 2 : 1) * SW_WIMG;
  TCB_CUDA(cudaFuncSetAttribute(wimg_build, cudaFuncAttributeMaxDynamicSharedMemorySize, wsm));
  for (long long c0 = 0; c0 < C; c0 += 1 << 30) {
    const unsigned nb = (unsigned)std::min<long long>(C - c0, 1 << 30);
    wimg_build<<<nb, SW_THREADS, wsm>>>(h->cs, h->rtab, h->etab, h->sw_toffs, h->sw_tlist,
                                        chunk_of + c0, ntx, geo,
                                        h->sw_whi + (size_t)c0 * (img / 16),
                                        with_lo ? h->sw_wlo + (size_t)c0 * (img / 16) : nullptr,
                                        h->sw_vidx + (size_t)c0 * SW_K);
  }
  count_launch(2);
  cudaError_t e = cudaDeviceSynchronize();
  cudaFree(chunk_of);
  if (e != cudaSuccess) {
    set_error("tcb_fourierrec_set_gridding: weight tables failed: %s", cudaGetErrorString(e));
    return TCB_ERR_CUDA;
  }
  TCB_CUDA(cudaFuncSetAttribute(grid_sw<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SwCfg<128, true>::SMEM));
  TCB_CUDA(cudaFuncSetAttribute(grid_sw<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SwCfg<128, false>::SMEM));
  TCB_CUDA(cudaFuncSetAttribute(grid_sw<64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SwCfg<64, true>::SMEM));
  TCB_CUDA(cudaFuncSetAttribute(grid_sw<64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SwCfg<64, false>::SMEM));
  h->sw_nn = nn;
  h->sw_ntx = ntx;
  h->sw_ntiles = nt;
  h->sw_zgroups = zgroups;
  h->sw_chunks = C;
  h->sw_nonempty = 0;
  for (int t = 0; t < nt; t++) h->sw_nonempty += tch[t].y > 0;
  h->sw_lo = with_lo;
  return TCB_OK;
}

}  // namespace

extern "C" int tcb_fourierrec_create(tcb_fourierrec **out, size_t nproj, size_t nz,
                                     size_t n, const float *theta, int precision) {
  TCB_CHECK_ARG(out, "tcb_fourierrec_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(theta, "tcb_fourierrec_create: null theta");
  // n >= TX keeps a 9-cell footprint from reaching one tile through two
  // periodic images.
  TCB_CHECK_ARG(n >= (size_t)TX && n % 2 == 0 && n <= 32768,
                "tcb_fourierrec_create: n=%zu must be even and in [%d, 32768]", n, TX);
  TCB_CHECK_ARG(nproj >= 1 && nproj < (1u << 20), "tcb_fourierrec_create: bad nproj %zu",
                nproj);
  TCB_CHECK_ARG(nz >= 1, "tcb_fourierrec_create: nz must be >= 1");
  TCB_CHECK_ARG(nproj * nz < (1ull << 31) && nproj * n < (1ull << 31),
                "tcb_fourierrec_create: nproj*nz or nproj*n too large");
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
  geo.ntx = (int)ceil_div(2 * n, TX);
  geo.nty = (int)ceil_div(2 * n, TY);
  geo.mu = mu;
  geo.coeff0 = TCB_PI_F / (mu * (4 * n * n));
  geo.coeff1 = -TCB_PI_F * TCB_PI_F / mu;
  geo.scale = 4.0f / n;
  h->ntiles = geo.ntx * geo.nty;

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
  FR_ALLOC(h->toffs, (h->ntiles + 1) * sizeof(long long));
  FR_ALLOC(h->boffs, ((size_t)h->ntiles * NREG + 1) * sizeof(long long));
  FR_ALLOC(h->grid, nz * 4 * n * n * sizeof(float2));
  FR_ALLOC(h->dtab, n * sizeof(float4));
  if (precision == TCB_FLOAT16) FR_ALLOC(h->g32, nz * nproj * n * sizeof(float2));
#undef FR_ALLOC

  // Tiles ordered by distance of their centre from the grid origin.
  std::vector<int> order(h->ntiles);
  std::vector<float> dist(h->ntiles);
  for (int t = 0; t < h->ntiles; t++) {
    order[t] = t;
    float cx = (t % geo.ntx) * TX + 0.5f * TX - (float)n;
    float cy = (t / geo.ntx) * TY + 0.5f * TY - (float)n;
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
  deapod_terms<<<ceil_div(n, 256), 256>>>(h->dtab, (int)n);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_error("tcb_fourierrec_create: table setup failed: %s", cudaGetErrorString(e));
    return fail(TCB_ERR_CUDA);
  }
  int st = build_lists(h);
  if (st != TCB_OK) return fail(st);
  e = cudaFuncSetAttribute(grid_blocks<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(GridSmem<16>));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(grid_blocks<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(GridSmem<8>));
  if (e != cudaSuccess) {
    set_error("tcb_fourierrec_create: smem attribute failed: %s", cudaGetErrorString(e));
    return fail(TCB_ERR_CUDA);
  }
  int len1[1] = {(int)n};
  cufftResult r = cufftPlanMany(&h->plan1d, 1, len1, nullptr, 1, 0, nullptr, 1, 0,
                                CUFFT_C2C, (int)(nproj * nz));
  int len2[2] = {(int)(2 * n), (int)(2 * n)};
  // The deapodization reads only rows and columns [n/2, 3n/2 + 1) of the
  // inverse 2D transform, so the 2D inverse FFT is pruned.  For a
  // power-of-two 2n in [256, 8192] the library's own FFT runs it: a row pass
  // over all 2n rows that writes only the n kept columns, then a column pass
  // over those n columns with the deapodization fused into its last stage
  // (2048-slice volume at 2n = 4096: 87 ms, against 128 ms for cuFFT's
  // pruned passes plus a deapodization kernel).  Other sizes use cuFFT:
  // rows over all 2n rows, then columns over the n kept columns.
  // TCB_FOURIERREC_FFT=cufft forces cuFFT, =own_cf the own FFT with the
  // column pass first; TCB_FOURIERREC_FULL_FFT2D=1 selects one full cuFFT
  // 2D transform.
  const char *full = getenv("TCB_FOURIERREC_FULL_FFT2D");
  const char *fsel = getenv("TCB_FOURIERREC_FFT");
  h->pruned = !(full && full[0] == '1');
  const size_t N2 = 2 * n;
  const bool own_sel = !(fsel && strcmp(fsel, "cufft") == 0);
  if (h->pruned && own_sel && N2 >= 256 && N2 <= 8192 &&
      (N2 & (N2 - 1)) == 0) {
    const std::vector<float2> twh = fftk::twiddle_table((int)N2);
    if (cudaMalloc(&h->tw, twh.size() * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&h->t1, nz * n * N2 * sizeof(float2)) != cudaSuccess) {
      cudaGetLastError();
      set_error("tcb_fourierrec_create: out of device memory for the FFT buffers");
      return fail(TCB_ERR_OUT_OF_MEMORY);
    }
    e = cudaMemcpy(h->tw, twh.data(), twh.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      switch (N2) {
        case 256: e = own_fft_attrs<256>(); break;
        case 512: e = own_fft_attrs<512>(); break;
        case 1024: e = own_fft_attrs<1024>(); break;
        case 2048: e = own_fft_attrs<2048>(); break;
        case 4096: e = own_fft_attrs<4096>(); break;
        default: e = own_fft_attrs<8192>(); break;
      }
    }
    if (e != cudaSuccess) {
      set_error("tcb_fourierrec_create: FFT setup failed: %s", cudaGetErrorString(e));
      return fail(TCB_ERR_CUDA);
    }
    h->own_n = (int)N2;
    // columns per block of the column pass: a power of two up to
    // cols_per_block (TCB_FOURIERREC_FFT_CPC tunes it)
    h->own_rows_first = !(fsel && strcmp(fsel, "own_cf") == 0);
    h->own_cpc = cols_per_block((int)N2);
    // TCB_FOURIERREC_T1_GW=4/8/16 sets the row-pass output grouping
    if (const char *c = getenv("TCB_FOURIERREC_T1_GW")) {
      const int v = atoi(c);
      if (v == 4 || v == 8 || v == 16) h->t1_gw = v;
    }
    if (const char *c = getenv("TCB_FOURIERREC_FFT_CPC")) {
      const int v = atoi(c);
      if (v >= 1 && v <= h->own_cpc && (v & (v - 1)) == 0) h->own_cpc = v;
    }
  }
  if (r == CUFFT_SUCCESS && !h->pruned)
    r = cufftPlanMany(&h->plan2d, 2, len2, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, (int)nz);
  if (r == CUFFT_SUCCESS && h->pruned && !h->own_n) {
    int lr[1] = {(int)(2 * n)};
    r = cufftPlanMany(&h->plan_rows, 1, lr, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C,
                      (int)(2 * n * nz));
    int emb[1] = {(int)(2 * n)};
    if (r == CUFFT_SUCCESS)
      r = cufftPlanMany(&h->plan_cols, 1, lr, emb, (int)(2 * n), 1, emb, (int)(2 * n), 1,
                        CUFFT_C2C, (int)n);
  }
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

// Sample positions and footprint origins exactly as the gridding kernels use
// them (sample_pos), one per (angle p, radial index i), in takexy's layout
// [p * n + i].
__global__ void sample_positions_kernel(float *__restrict__ x, float *__restrict__ y,
                                        int *__restrict__ fx, int *__restrict__ fy,
                                        const float2 *__restrict__ cs,
                                        const float *__restrict__ rtab, int n, int nproj) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)n * nproj) return;
  float x0, y0;
  int ox, oy;
  sample_pos(cs, rtab, (int)(i / n), (int)(i % n), (float)(2 * n), x0, y0, ox, oy);
  x[i] = x0;
  y[i] = y0;
  fx[i] = ox;
  fy[i] = oy;
}

extern "C" int tcb_fourierrec_sample_positions(tcb_fourierrec *h, float *x, float *y, int *fx,
                                               int *fy, void *stream) {
  TCB_CHECK_ARG(h && x && y && fx && fy, "tcb_fourierrec_sample_positions: null pointer");
  TCB_CHECK_ARG(h->grid, "tcb_fourierrec_sample_positions: handle was freed");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t total = h->n * h->nproj;
  sample_positions_kernel<<<ceil_div(total, 256), 256, 0, s>>>(x, y, fx, fy, h->cs, h->rtab,
                                                               (int)h->n, (int)h->nproj);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

extern "C" int tcb_fourierrec_set_pairs_per_block(tcb_fourierrec *h, int pairs) {
  TCB_CHECK_ARG(h, "tcb_fourierrec_set_pairs_per_block: null handle");
  TCB_CHECK_ARG(pairs == 0 || pairs == 2 || pairs == 4 || pairs == 8 || pairs == 16,
                "tcb_fourierrec_set_pairs_per_block: pairs must be 0, 2, 4, 8 or 16");
  h->zblock = pairs;
  return TCB_OK;
}

extern "C" int tcb_fourierrec_set_input_spectrum(tcb_fourierrec *h, int on) {
  TCB_CHECK_ARG(h, "tcb_fourierrec_set_input_spectrum: null handle");
  TCB_CHECK_ARG(h->grid, "tcb_fourierrec_set_input_spectrum: handle was freed");
  TCB_CHECK_ARG(h->precision == TCB_FLOAT32,
                "tcb_fourierrec_set_input_spectrum: FLOAT32 handles only");
  h->spectrum_in = on != 0;
  return TCB_OK;
}

extern "C" int tcb_fourierrec_set_gridding(tcb_fourierrec *h, int mode) {
  TCB_CHECK_ARG(h, "tcb_fourierrec_set_gridding: null handle");
  TCB_CHECK_ARG(h->grid, "tcb_fourierrec_set_gridding: handle was freed");
  TCB_CHECK_ARG(mode == TCB_GRID_FP32 || mode == TCB_GRID_TENSOR ||
                    mode == TCB_GRID_TENSOR_FP32 || mode == TCB_GRID_TENSOR_STREAM,
                "tcb_fourierrec_set_gridding: unknown mode %d", mode);
  if (mode == TCB_GRID_TENSOR_FP32 || mode == TCB_GRID_TENSOR_STREAM) {
    TCB_CHECK_ARG(h->precision == TCB_FLOAT32,
                  "tcb_fourierrec_set_gridding: streamed tensor gridding needs a FLOAT32 handle");
    TCB_CHECK_ARG(h->nproj * h->n < (size_t)INT32_MAX,
                  "tcb_fourierrec_set_gridding: nproj * n too large for the tensor gridding");
    const bool want_lo = mode == TCB_GRID_TENSOR_FP32;
    if (h->sw_nn == 0 || (want_lo && !h->sw_lo)) {
      if (h->sw_nn) {  // rebuild with lo images
        cudaFree(h->sw_whi);
        cudaFree(h->sw_wlo);
        h->sw_whi = h->sw_wlo = nullptr;
      }
      const int st = sw_build(h, want_lo);
      if (st != TCB_OK) return st;
    }
    if (!h->amax) {
      if (cudaMalloc(&h->amax, sizeof(unsigned)) != cudaSuccess ||
          cudaMalloc(&h->tc_err, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        set_error("tcb_fourierrec_set_gridding: out of device memory");
        return TCB_ERR_OUT_OF_MEMORY;
      }
      TCB_CUDA(cudaMemset(h->tc_err, 0, sizeof(int)));
    }
    h->grid_mode = mode;
    return TCB_OK;
  }
  if (mode == TCB_GRID_TENSOR && !h->amax) {
    TCB_CHECK_ARG(h->nproj * h->n < (size_t)INT32_MAX,
                  "tcb_fourierrec_set_gridding: nproj * n too large for the tensor gridding");
    long long total = 0;  // listed (tile, sample) entries
    TCB_CUDA(cudaMemcpy(&total, h->toffs + h->ntiles, sizeof(long long),
                        cudaMemcpyDeviceToHost));
    if (cudaMalloc(&h->amax, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&h->tc_err, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->trec, ((size_t)total + 1) * TC_REC * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      set_error("tcb_fourierrec_set_gridding: out of device memory (%lld records)", total);
      return TCB_ERR_OUT_OF_MEMORY;
    }
    TCB_CUDA(cudaMemset(h->tc_err, 0, sizeof(int)));
    TCB_CUDA(cudaFuncSetAttribute(grid_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TC_SMEM));
    tile_records<<<(unsigned)h->ntiles, 256>>>(h->cs, h->rtab, h->etab, h->toffs, h->tlist,
                                               h->geo, h->trec);
    count_launch();
    TCB_CUDA(cudaDeviceSynchronize());
  }
  h->grid_mode = mode;
  return TCB_OK;
}

extern "C" int tcb_fourierrec_set_output(tcb_fourierrec *h, int precision) {
  TCB_CHECK_ARG(h, "tcb_fourierrec_set_output: null handle");
  TCB_CHECK_ARG(precision == TCB_FLOAT32 || precision == TCB_FLOAT16,
                "tcb_fourierrec_set_output: unknown precision %d", precision);
  h->out_f16 = precision == TCB_FLOAT16;
  return TCB_OK;
}

extern "C" int tcb_fourierrec_status(tcb_fourierrec *h, int *timed_out) {
  TCB_CHECK_ARG(h && timed_out, "tcb_fourierrec_status: null pointer");
  *timed_out = 0;
  if (h->tc_err) TCB_CUDA(cudaMemcpy(timed_out, h->tc_err, sizeof(int), cudaMemcpyDeviceToHost));
  return TCB_OK;
}

extern "C" int tcb_fourierrec_destroy(tcb_fourierrec *h) {
  if (!h) return TCB_OK;
  fr_release(h);
  delete h;
  return TCB_OK;
}
