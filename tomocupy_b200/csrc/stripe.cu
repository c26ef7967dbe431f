// Fourier-wavelet ring removal (remove_stripe_fw).
//
// Same algorithm as the reference (src/tomocupy/processing/remove_stripe.py:
// _reflect/_mypad 51-84, afb1d 86-128, sfb1d 131-155, DWTForward 157-200,
// DWTInverse 202-246, remove_stripe_fw 253-293): the sinograms, padded along
// the angles to nproj + nproj/8 with zeros, go through `level` 2D DWT levels
// (stride-2 correlation with the reversed analysis filters along the
// detector, then along the angles, half-sample symmetric extension, output
// length floor((N + L - 1)/2)); at every level the band that is high-pass
// along the detector and low-pass along the angles (vertical stripes) is
// Fourier transformed along the angles, multiplied by
// -expm1(-k^2 / (2 sigma^2)) and transformed back; the inverse DWT (stride-2
// transposed convolution with the synthesis filters, cropped by L-2 on both
// sides) rebuilds the sinograms.
//
// Every tap is accumulated in the reference's order with explicit
// round-to-nearest multiplies and adds (no contraction), so the wavelet
// stages reproduce its float32 arithmetic; the band FFTs use cuFFT.
// B200 design: one kernel per filter pass over all slices of the chunk,
// both output channels of a pass from one read of the input window, the
// pyramid kept in HBM.  The damping y = irfft(rfft(x) (1 - g)) along the
// angles equals x - (1/H) sum_k g_k X_k e^{2 pi i k q / H}, and the
// Gaussian g_k = exp(-v_k^2 / (2 sigma^2)) (v_k = k, or k + 1/2 for even H,
// as the reference's ifftshifted grid gives) is below 1e-12 beyond a few
// modes (k <= 7 for sigma = 1): the band is damped in place by projecting
// each column onto those modes (sums of x cos, x sin) and subtracting the
// low-pass, one read and one write of the band, no transposes, no FFTs.
// Levels whose band is too short for the modes, or sigmas that need more
// than 32 (TCB_FW_DAMP=cufft forces it), transpose the band and use cuFFT
// R2C / C2R with 1/N folded into the damping factors.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "common.cuh"

namespace tcb {
namespace sw {

constexpr int MAXL = 64;

struct Taps {
  float h0[MAXL], h1[MAXL];  // analysis: dec_lo, dec_hi reversed
  float g0[MAXL], g1[MAXL];  // synthesis: rec_lo, rec_hi
  int L;
};

__device__ __forceinline__ int reflect(int m, int n) {
  int p = 2 * n;
  m %= p;
  if (m < 0) m += p;
  return m >= n ? p - 1 - m : m;
}

// The filter-bank kernels keep the reference's per-tap operation order
// (round-to-nearest multiply then add, tap by tap), so results are
// bit-identical; the taps live in shared memory and the symmetric reflection
// is only evaluated for outputs whose support crosses an edge.
struct SmemTaps {
  float a[MAXL], b[MAXL];
};

__device__ __forceinline__ void load_taps(SmemTaps &st, const float *a, const float *b, int L) {
  for (int k = threadIdx.x + threadIdx.y * blockDim.x; k < L; k += blockDim.x * blockDim.y) {
    st.a[k] = a[k];
    st.b[k] = b[k];
  }
  __syncthreads();
}

// afb1d along the last axis: x [B][H][W] (row stride sx, slice stride sz) ->
// out [B][2][H][Wo] (lo, hi).
__global__ void afb_rows(const float *__restrict__ x, long long sz, int sx, float *__restrict__ out,
                         int B, int H, int W, int Wo, int padl, const Taps *__restrict__ taps) {
  __shared__ SmemTaps st;
  const int L = taps->L;
  load_taps(st, taps->h0, taps->h1, L);
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = (long long)B * H * Wo;
  if (idx >= total) return;
  int j = (int)(idx % Wo);
  long long r = idx / Wo;
  int h = (int)(r % H);
  int b = (int)(r / H);
  const float *row = x + b * sz + (long long)h * sx;
  const int base = 2 * j - padl;
  float v = row[base >= 0 && base < W ? base : reflect(base, W)];
  float lo = __fmul_rn(st.a[0], v), hi = __fmul_rn(st.b[0], v);
  if (base >= 0 && base + L <= W) {
    for (int k = 1; k < L; k++) {
      v = row[base + k];
      lo = __fadd_rn(lo, __fmul_rn(st.a[k], v));
      hi = __fadd_rn(hi, __fmul_rn(st.b[k], v));
    }
  } else {
    for (int k = 1; k < L; k++) {
      v = row[reflect(base + k, W)];
      lo = __fadd_rn(lo, __fmul_rn(st.a[k], v));
      hi = __fadd_rn(hi, __fmul_rn(st.b[k], v));
    }
  }
  long long o = (((long long)b * 2) * H + h) * Wo + j;
  out[o] = lo;
  out[o + (long long)H * Wo] = hi;
}

// afb1d along the rows axis for both channels: in [B][2][H][W] ->
// out [B][4][Ho][W] (channel c -> 2c lo, 2c+1 hi).
__global__ void afb_cols(const float *__restrict__ in, float *__restrict__ out, int B, int H,
                         int W, int Ho, int padl, const Taps *__restrict__ taps) {
  __shared__ SmemTaps st;
  const int L = taps->L;
  load_taps(st, taps->h0, taps->h1, L);
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = (long long)B * 2 * Ho * W;
  if (idx >= total) return;
  int j = (int)(idx % W);
  long long r = idx / W;
  int i = (int)(r % Ho);
  long long bc = r / Ho;  // b*2 + c
  const float *col = in + bc * H * W + j;
  const int base = 2 * i - padl;
  float v = col[(long long)(base >= 0 && base < H ? base : reflect(base, H)) * W];
  float lo = __fmul_rn(st.a[0], v), hi = __fmul_rn(st.b[0], v);
  if (base >= 0 && base + L <= H) {
    const float *c0 = col + (long long)base * W;
    for (int k = 1; k < L; k++) {
      v = c0[(long long)k * W];
      lo = __fadd_rn(lo, __fmul_rn(st.a[k], v));
      hi = __fadd_rn(hi, __fmul_rn(st.b[k], v));
    }
  } else {
    for (int k = 1; k < L; k++) {
      v = col[(long long)reflect(base + k, H) * W];
      lo = __fadd_rn(lo, __fmul_rn(st.a[k], v));
      hi = __fadd_rn(hi, __fmul_rn(st.b[k], v));
    }
  }
  long long b = bc / 2, c = bc % 2;
  long long o = ((b * 4 + 2 * c) * Ho + i) * W + j;
  out[o] = lo;
  out[o + (long long)Ho * W] = hi;
}

// sfb1d along the rows axis: channel 0 = synth(lo0, hi0), 1 = synth(lo1, hi1)
// with lo0 = LL (stride sll), hi0 = band0, lo1 = band1, hi1 = band2 of a
// [B][4][Hi][Wb] pyramid level; LL may be cropped (Hi, W used).  Output
// [B][2][Ho][W], Ho = 2 Hi - L + 2.
__global__ void sfb_cols(const float *__restrict__ y, long long bstride, int Hi, int Wb, int W,
                         float *__restrict__ out, int B, int Ho, const Taps *__restrict__ taps) {
  __shared__ SmemTaps st;
  const int L = taps->L;
  load_taps(st, taps->g0, taps->g1, L);
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = (long long)B * 2 * Ho * W;
  if (idx >= total) return;
  int j = (int)(idx % W);
  long long r = idx / W;
  int t = (int)(r % Ho);
  long long bc = r / Ho;
  int b = (int)(bc / 2), c = (int)(bc % 2);
  const long long plane = (long long)Hi * Wb;
  const float *base = y + b * bstride;
  const float *lo = base + (c == 0 ? 0 : 2) * plane + j;  // LL or band1 (HL)
  const float *hi = base + (c == 0 ? 1 : 3) * plane + j;  // band0 (LH) or band2 (HH)
  int tt = t + L - 2;  // position in the uncropped output
  float acc = 0.f;
  for (int k = tt & 1; k < L; k += 2) {
    int h = (tt - k) >> 1;
    if (h < 0 || h >= Hi) continue;
    float v = __fadd_rn(__fmul_rn(st.a[k], lo[(long long)h * Wb]),
                        __fmul_rn(st.b[k], hi[(long long)h * Wb]));
    acc = __fadd_rn(acc, v);
  }
  out[(bc * Ho + t) * W + j] = acc;
}

// sfb1d along the last axis: in [B][2][H][Wi] -> out rows (b, h) of width
// Wo = 2 Wi - L + 2, written to dst[b*dsz + h*dsx + w] for h < Hd, w < Wd.
__global__ void sfb_rows(const float *__restrict__ in, int H, int Wi, float *__restrict__ dst,
                         long long dsz, int dsx, int Hd, int Wd, int B,
                         const Taps *__restrict__ taps) {
  __shared__ SmemTaps st;
  const int L = taps->L;
  load_taps(st, taps->g0, taps->g1, L);
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = (long long)B * Hd * Wd;
  if (idx >= total) return;
  int w = (int)(idx % Wd);
  long long r = idx / Wd;
  int h = (int)(r % Hd);
  int b = (int)(r / Hd);
  const float *lo = in + (((long long)b * 2) * H + h) * Wi;
  const float *hi = lo + (long long)H * Wi;
  int tt = w + L - 2;
  float acc = 0.f;
  for (int k = tt & 1; k < L; k += 2) {
    int q = (tt - k) >> 1;
    if (q < 0 || q >= Wi) continue;
    float v = __fadd_rn(__fmul_rn(st.a[k], lo[q]), __fmul_rn(st.b[k], hi[q]));
    acc = __fadd_rn(acc, v);
  }
  dst[b * dsz + (long long)h * dsx + w] = acc;
}

// ---- register-blocked filter banks for the supported filter lengths ------
// Same outputs, bit for bit, as the kernels above (every output keeps its
// multiply-then-add tap order); the taps come from the kernel parameter
// space (constant-bank operands of the multiplies, fully unrolled), and each
// input value is read once per thread window instead of once per tap.
struct TapPair {
  float a[MAXL], b[MAXL];
};

// afb1d along the last axis.  RB rows per block staged in shared memory with
// the symmetric extension applied (smem[u] = x[reflect(u - padl)]); output j
// reads smem[2j + k], k < L, as L/2 float2 loads (conflict-free).
template <int L>
__global__ void __launch_bounds__(256) afb_rows_t(const float *__restrict__ x, long long sz,
                                                  int sx, float *__restrict__ out, int B, int H,
                                                  int W, int Wo, int padl, int RB, int SW,
                                                  const __grid_constant__ TapPair t) {
  extern __shared__ float2 srow2[];
  float *srow = reinterpret_cast<float *>(srow2);
  const long long row0 = (long long)blockIdx.x * RB;
  const long long nrows = (long long)B * H;
  const int nr = (int)min((long long)RB, nrows - row0);
  for (int r = 0; r < nr; r++) {
    const long long row = row0 + r;
    const long long b = row / H, h = row - b * H;
    const float *xr = x + b * sz + h * sx;
    float *sr = srow + r * SW;
    for (int u = threadIdx.x; u < SW; u += blockDim.x) {
      const int m = u - padl;
      sr[u] = xr[m >= 0 && m < W ? m : reflect(m, W)];
    }
  }
  __syncthreads();
  constexpr int RO = 4;                 // outputs per thread
  constexpr int NV = 2 * RO + L - 2;    // their input window
  const int ngrp = (Wo + RO - 1) / RO;
  for (int e = threadIdx.x; e < nr * ngrp; e += blockDim.x) {
    const int r = e / ngrp, j0 = (e - r * ngrp) * RO;
    const float2 *p = srow2 + (r * SW) / 2 + j0;  // smem[2 j0 + u] = window u
    float v[NV];
#pragma unroll
    for (int q = 0; q < NV / 2; q++) {
      const float2 w = p[q];
      v[2 * q] = w.x;
      v[2 * q + 1] = w.y;
    }
    float lo[RO], hi[RO];
#pragma unroll
    for (int o = 0; o < RO; o++) {
      lo[o] = __fmul_rn(t.a[0], v[2 * o]);
      hi[o] = __fmul_rn(t.b[0], v[2 * o]);
    }
#pragma unroll
    for (int k = 1; k < L; k++) {
      const float ak = t.a[k], bk = t.b[k];
#pragma unroll
      for (int o = 0; o < RO; o++) {
        lo[o] = __fadd_rn(lo[o], __fmul_rn(ak, v[2 * o + k]));
        hi[o] = __fadd_rn(hi[o], __fmul_rn(bk, v[2 * o + k]));
      }
    }
    const long long row = row0 + r;
    const long long b = row / H, h = row - b * H;
    float *o0 = out + ((b * 2) * H + h) * Wo;
    float *o1 = o0 + (long long)H * Wo;
#pragma unroll
    for (int o = 0; o < RO; o++)
      if (j0 + o < Wo) {
        o0[j0 + o] = lo[o];
        o1[j0 + o] = hi[o];
      }
  }
}

// Column kernels: a block is a tile of 32 columns x (8 * RO) output rows of
// one channel plane; the input rows of the tile are staged in shared memory
// (one coalesced pass), then thread (tx, ty) computes column tx, rows
// ty*RO .. ty*RO + RO - 1 of the tile from a register window.
constexpr int CT_X = 32, CT_Y = 8;

// afb1d along the rows axis: in [B][2][H][W] -> out [B][4][Ho][W]; thread =
// column j and RO consecutive output rows, its 2 RO + L - 2 input rows held
// in registers (read through L1: the windows of neighbouring row groups
// overlap).
template <int L, int RO>
__global__ void __launch_bounds__(128) afb_cols_t(const float *__restrict__ in,
                                                  float *__restrict__ out, int B, int H, int W,
                                                  int Ho, int padl,
                                                  const __grid_constant__ TapPair t) {
  const int ncolb = (W + blockDim.x - 1) / blockDim.x;
  const int ngrp = (Ho + RO - 1) / RO;
  const long long blk = blockIdx.x;
  const int j = (int)(blk % ncolb) * blockDim.x + threadIdx.x;
  const long long rest = blk / ncolb;
  const long long bc = rest / ngrp;
  const int i0 = (int)(rest - bc * ngrp) * RO;
  if (j >= W) return;
  const float *col = in + bc * H * W + j;
  constexpr int NV = 2 * RO + L - 2;
  float v[NV];
  const int r0 = 2 * i0 - padl;
  if (r0 >= 0 && r0 + NV <= H) {
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = col[(long long)(r0 + q) * W];
  } else {
#pragma unroll
    for (int q = 0; q < NV; q++) {
      const int rr = r0 + q;
      v[q] = col[(long long)(rr >= 0 && rr < H ? rr : reflect(rr, H)) * W];
    }
  }
  const long long b = bc / 2, c = bc % 2;
  float *o0 = out + ((b * 4 + 2 * c) * Ho) * (long long)W + j;
  float *o1 = o0 + (long long)Ho * W;
  float lo[RO], hi[RO];
#pragma unroll
  for (int r = 0; r < RO; r++) {
    lo[r] = __fmul_rn(t.a[0], v[2 * r]);
    hi[r] = __fmul_rn(t.b[0], v[2 * r]);
  }
#pragma unroll
  for (int k = 1; k < L; k++) {
    const float ak = t.a[k], bk = t.b[k];
#pragma unroll
    for (int r = 0; r < RO; r++) {
      lo[r] = __fadd_rn(lo[r], __fmul_rn(ak, v[2 * r + k]));
      hi[r] = __fadd_rn(hi[r], __fmul_rn(bk, v[2 * r + k]));
    }
  }
#pragma unroll
  for (int r = 0; r < RO; r++)
    if (i0 + r < Ho) {
      o0[(long long)(i0 + r) * W] = lo[r];
      o1[(long long)(i0 + r) * W] = hi[r];
    }
}

// One synthesis output: acc over k of the reference's parity (k = tt & 1,
// tt & 1 + 2, ...), h = (tt - k)/2 skipped outside [0, Hi).  Windows lo/hi
// hold h = hb + idx; RO consecutive outputs with tt0 even (L even), so
// h = hb + L/2 + (r - k)/2.
template <int L, int RO, bool CHECK>
__device__ __forceinline__ void synth_outputs(const float (&lo)[L / 2 + RO / 2],
                                              const float (&hi)[L / 2 + RO / 2], int hb, int Hi,
                                              const TapPair &t, float (&acc)[RO]) {
#pragma unroll
  for (int r = 0; r < RO; r++) acc[r] = 0.f;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const float ak = t.a[k], bk = t.b[k];
#pragma unroll
    for (int r = k & 1; r < RO; r += 2) {
      const int idx = (r - k) / 2 + L / 2;  // h - hb
      if (CHECK) {
        const int h = hb + idx;
        if (h < 0 || h >= Hi) continue;
      }
      const float vv = __fadd_rn(__fmul_rn(ak, lo[idx]), __fmul_rn(bk, hi[idx]));
      acc[r] = __fadd_rn(acc[r], vv);
    }
  }
}

// sfb1d along the rows axis (see sfb_cols): tile rows t0.. (t0 a multiple
// of 8 * RO, so every thread's first output row is even).
template <int L, int RO>
__global__ void __launch_bounds__(CT_X *CT_Y) sfb_cols_t(const float *__restrict__ y,
                                                         long long bstride, int Hi, int Wb, int W,
                                                         float *__restrict__ out, int B, int Ho,
                                                         const __grid_constant__ TapPair t) {
  static_assert(L % 2 == 0 && RO % 2 == 0, "even filter length and output block");
  constexpr int TR = CT_Y * RO;
  constexpr int NW = L / 2 + RO / 2;       // window per thread
  constexpr int NT = TR / 2 + L / 2;       // window per tile
  __shared__ float tlo[NT][CT_X], thi[NT][CT_X];
  const int ncolb = (W + CT_X - 1) / CT_X;
  const int ngrp = (Ho + TR - 1) / TR;
  const long long blk = blockIdx.x;
  const int cb = (int)(blk % ncolb);
  const long long rest = blk / ncolb;
  const long long bc = rest / ngrp;
  const int t0 = (int)(rest - bc * ngrp) * TR;
  const int tx = threadIdx.x % CT_X, ty = threadIdx.x / CT_X;
  const int j = cb * CT_X + tx;
  const int b = (int)(bc / 2), c = (int)(bc % 2);
  const long long plane = (long long)Hi * Wb;
  const float *base = y + b * bstride;
  const float *lop = base + (c == 0 ? 0 : 2) * plane + j;  // LL or band1 (HL)
  const float *hip = base + (c == 0 ? 1 : 3) * plane + j;  // band0 (LH) or band2 (HH)
  const int hbt = (t0 + L - 2) / 2 - L / 2;  // h of tile window index 0
  for (int q = ty; q < NT; q += CT_Y) {
    const int h = hbt + q;
    const bool ok = j < W && h >= 0 && h < Hi;
    tlo[q][tx] = ok ? lop[(long long)h * Wb] : 0.f;
    thi[q][tx] = ok ? hip[(long long)h * Wb] : 0.f;
  }
  __syncthreads();
  if (j >= W) return;
  const int hb = hbt + ty * (RO / 2);
  float lo[NW], hi[NW];
#pragma unroll
  for (int q = 0; q < NW; q++) {
    lo[q] = tlo[ty * (RO / 2) + q][tx];
    hi[q] = thi[ty * (RO / 2) + q][tx];
  }
  float acc[RO];
  if (hb >= 0 && hb + NW <= Hi)
    synth_outputs<L, RO, false>(lo, hi, hb, Hi, t, acc);
  else
    synth_outputs<L, RO, true>(lo, hi, hb, Hi, t, acc);
  const int tt0 = t0 + ty * RO;
#pragma unroll
  for (int r = 0; r < RO; r++)
    if (tt0 + r < Ho) out[(bc * Ho + tt0 + r) * W + j] = acc[r];
}

// sfb1d along the last axis (see sfb_rows): thread = RO consecutive outputs
// w0.. of one row (w0 a multiple of RO), windows read through L1.
template <int L, int RO>
__global__ void __launch_bounds__(128) sfb_rows_t(const float *__restrict__ in, int H, int Wi,
                                                  float *__restrict__ dst, long long dsz, int dsx,
                                                  int Hd, int Wd, int B,
                                                  const __grid_constant__ TapPair t) {
  const int ngrp = (Wd + RO - 1) / RO;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)B * Hd * ngrp) return;
  const int w0 = (int)(g % ngrp) * RO;
  const long long rowi = g / ngrp;
  const int h = (int)(rowi % Hd);
  const int b = (int)(rowi / Hd);
  const float *lop = in + (((long long)b * 2) * H + h) * Wi;
  const float *hip = lop + (long long)H * Wi;
  constexpr int NW = L / 2 + RO / 2;
  const int hb = (w0 + L - 2) / 2 - L / 2;
  float lo[NW], hi[NW];
#pragma unroll
  for (int q = 0; q < NW; q++) {
    const int qq = hb + q;
    const bool ok = qq >= 0 && qq < Wi;
    lo[q] = ok ? lop[qq] : 0.f;
    hi[q] = ok ? hip[qq] : 0.f;
  }
  float acc[RO];
  if (hb >= 0 && hb + NW <= Wi)
    synth_outputs<L, RO, false>(lo, hi, hb, Wi, t, acc);
  else
    synth_outputs<L, RO, true>(lo, hi, hb, Wi, t, acc);
  float *d = dst + b * dsz + (long long)h * dsx;
#pragma unroll
  for (int r = 0; r < RO; r++)
    if (w0 + r < Wd) d[w0 + r] = acc[r];
}

// [B][R][C] <-> [B][C][R] (32x32 tiles)
__global__ void transpose_bands(const float *__restrict__ in, long long istride,
                                float *__restrict__ out, long long ostride, int R, int C) {
  __shared__ float t[32][33];
  int b = blockIdx.z;
  int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const float *src = in + b * istride;
  float *dst = out + b * ostride;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int r = r0 + k, c = c0 + threadIdx.x;
    if (r < R && c < C) t[k][threadIdx.x] = src[(long long)r * C + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int c = c0 + k, r = r0 + threadIdx.x;
    if (r < R && c < C) dst[(long long)c * R + r] = t[threadIdx.x][k];
  }
}

__global__ void damp_kernel(float2 *__restrict__ spec, const float *__restrict__ damp, int nc,
                            long long total) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  float d = damp[i % nc];
  float2 v = spec[i];
  spec[i] = make_float2(v.x * d, v.y * d);
}

// Damping by the low Fourier modes, in place on band [B][H][W] (slice
// stride bstride): a block takes 32 adjacent columns (threadIdx.x) of one
// slice, 8 row phases (threadIdx.y).  cs[k * H + q] = (cos, sin)(2 pi k q / H)
// and gw[k] = g_k / H (k = 0) or 2 g_k / H (k >= 1, the mode and its mirror
// H - k).  Pass 1 sums A_k = sum_q x_q cos, S_k = sum_q x_q sin per column;
// pass 2 writes x_q - sum_k gw_k (A_k cos + S_k sin).
constexpr int DM_R = 8;

template <int V1>
__global__ void __launch_bounds__(32 * DM_R)
    damp_modes(float *__restrict__ band, long long bstride, int H, int W,
               const float2 *__restrict__ cs, const float *__restrict__ gw) {
  __shared__ float red[DM_R][V1][32];
  const int w = blockIdx.x * 32 + threadIdx.x, r = threadIdx.y;
  float *col = band + (long long)blockIdx.y * bstride + w;
  const bool on = w < W;
  float A[V1], S[V1];
#pragma unroll
  for (int k = 0; k < V1; k++) A[k] = S[k] = 0.f;
  if (on)
    for (int q = r; q < H; q += DM_R) {
      const float x = col[(long long)q * W];
#pragma unroll
      for (int k = 0; k < V1; k++) {
        const float2 t = __ldg(cs + k * H + q);
        A[k] = fmaf(x, t.x, A[k]);
        S[k] = fmaf(x, t.y, S[k]);
      }
    }
  // the 8 row phases' partial sums, cosine then sine terms through one buffer
#pragma unroll
  for (int k = 0; k < V1; k++) red[r][k][threadIdx.x] = A[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < V1; k++) {
    float a = 0.f;
#pragma unroll
    for (int j = 0; j < DM_R; j++) a += red[j][k][threadIdx.x];
    A[k] = a * __ldg(gw + k);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < V1; k++) red[r][k][threadIdx.x] = S[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < V1; k++) {
    float b = 0.f;
#pragma unroll
    for (int j = 0; j < DM_R; j++) b += red[j][k][threadIdx.x];
    S[k] = b * __ldg(gw + k);
  }
  if (!on) return;
  for (int q = r; q < H; q += DM_R) {
    float lp = 0.f;
#pragma unroll
    for (int k = 0; k < V1; k++) {
      const float2 t = __ldg(cs + k * H + q);
      lp = fmaf(A[k], t.x, fmaf(S[k], t.y, lp));
    }
    col[(long long)q * W] -= lp;
  }
}

}  // namespace sw
}  // namespace tcb

using namespace tcb;
using namespace tcb::sw;

struct tcb_stripe_fw {
  int nproj, nz, ni, level, nproj_pad, L;
  std::vector<int> H, W;  // level sizes: H[0] = nproj_pad, W[0] = ni
  std::vector<float *> Y; // per level [nz][4][H[k+1]][W[k+1]]
  std::vector<float *> damp;  // per level damping factors (with 1/H)
  std::vector<cufftHandle> r2c, c2r;
  std::vector<int> modes;     // per level: modes of the direct damping (0 = cuFFT)
  std::vector<float2 *> mcs;  // per level [modes][H] (cos, sin)(2 pi k q / H)
  std::vector<float *> mgw;   // per level [modes] weights
  float *tmp = nullptr;    // [nz][2][H][W] scratch
  float *bt = nullptr;     // transposed band scratch
  float2 *spec = nullptr;  // band spectrum scratch
  Taps *taps = nullptr;    // device copy
  size_t tmp_elems = 0;
  TapPair ana{}, syn{};    // by-value taps of the register-blocked kernels
};

namespace {
constexpr int FB_RO = 4;  // outputs per thread of the column / synthesis kernels

template <int L>
void launch_afb_rows(const tcb_stripe_fw *h, const float *x, long long xsz, int xsx, int B,
                     int Hk, int Wk, int Wo, int padl, cudaStream_t s) {
  const int SW = 2 * ((Wo + 3) / 4 * 4) + L - 2;  // windows of the last 4-output group
  const int RB = std::max(1, std::min(16, 1024 / Wo));
  const long long nb = ((long long)B * Hk + RB - 1) / RB;
  afb_rows_t<L><<<(unsigned)nb, 256, (size_t)RB * SW * sizeof(float), s>>>(
      x, xsz, xsx, h->tmp, B, Hk, Wk, Wo, padl, RB, SW, h->ana);
}

template <int L>
void launch_afb_cols(const tcb_stripe_fw *h, float *out, int B, int Hk, int Wo, int Ho, int padl,
                     cudaStream_t s) {
  const long long nb = (long long)ceil_div(Wo, 128) * (2LL * B) * ((Ho + FB_RO - 1) / FB_RO);
  afb_cols_t<L, FB_RO><<<(unsigned)nb, 128, 0, s>>>(h->tmp, out, B, Hk, Wo, Ho, padl, h->ana);
}

template <int L>
void launch_sfb_cols(const tcb_stripe_fw *h, const float *y, int Hi, int Wi, int B, int Hc,
                     cudaStream_t s) {
  const long long nb = (long long)ceil_div(Wi, CT_X) * (2LL * B) *
                       ((Hc + CT_Y * FB_RO - 1) / (CT_Y * FB_RO));
  sfb_cols_t<L, FB_RO><<<(unsigned)nb, CT_X * CT_Y, 0, s>>>(y, 4LL * Hi * Wi, Hi, Wi, Wi,
                                                            h->tmp, B, Hc, h->syn);
}

template <int L>
void launch_sfb_rows(const tcb_stripe_fw *h, int Hc, int Wi, float *dst, long long dsz, int Wd,
                     int Hrows, int B, cudaStream_t s) {
  const long long thr = (long long)B * Hrows * ((Wd + FB_RO - 1) / FB_RO);
  sfb_rows_t<L, FB_RO><<<(unsigned)ceil_div(thr, 128), 128, 0, s>>>(h->tmp, Hc, Wi, dst, dsz, Wd,
                                                                    Hrows, Wd, B, h->syn);
}

bool blocked_length(int L) { return L == 2 || L == 10 || L == 32; }
}  // namespace

static void fw_release(tcb_stripe_fw *h) {
  for (auto p : h->Y) cudaFree(p);
  for (auto p : h->damp) cudaFree(p);
  for (auto p : h->r2c) if (p) cufftDestroy(p);
  for (auto p : h->c2r) if (p) cufftDestroy(p);
  for (auto p : h->mcs) cudaFree(p);
  for (auto p : h->mgw) cudaFree(p);
  h->mcs.clear();
  h->mgw.clear();
  h->modes.clear();
  h->Y.clear();
  h->damp.clear();
  h->r2c.clear();
  h->c2r.clear();
  cudaFree(h->tmp);
  cudaFree(h->bt);
  cudaFree(h->spec);
  cudaFree(h->taps);
  h->tmp = h->bt = nullptr;
  h->spec = nullptr;
  h->taps = nullptr;
}

extern "C" int tcb_stripe_fw_create(tcb_stripe_fw **out, size_t nproj, size_t nz, size_t ni,
                                    int level, float sigma, const double *dec_lo,
                                    const double *dec_hi, const double *rec_lo,
                                    const double *rec_hi, int L) {
  TCB_CHECK_ARG(out, "tcb_stripe_fw_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 2 && nz >= 1 && ni >= 2 && level >= 1 && level <= 16,
                "tcb_stripe_fw_create: bad sizes");
  TCB_CHECK_ARG(L >= 2 && L <= MAXL && dec_lo && dec_hi && rec_lo && rec_hi,
                "tcb_stripe_fw_create: bad filter bank (L=%d)", L);
  TCB_CHECK_ARG(sigma > 0, "tcb_stripe_fw_create: sigma must be > 0");
  tcb_stripe_fw *h = new tcb_stripe_fw();
  h->nproj = (int)nproj;
  h->nz = (int)nz;
  h->ni = (int)ni;
  h->level = level;
  h->nproj_pad = (int)(nproj + nproj / 8);
  h->L = L;
  h->H.push_back(h->nproj_pad);
  h->W.push_back((int)ni);
  for (int k = 0; k < level; k++) {
    h->H.push_back((h->H[k] + L - 1) / 2);
    h->W.push_back((h->W[k] + L - 1) / 2);
  }
  auto fail = [&](int code, const char *what) {
    set_error("tcb_stripe_fw_create: %s", what);
    fw_release(h);
    delete h;
    return code;
  };
  Taps t{};
  t.L = L;
  for (int k = 0; k < L; k++) {  // float32 taps, analysis filters reversed
    t.h0[k] = (float)dec_lo[L - 1 - k];
    t.h1[k] = (float)dec_hi[L - 1 - k];
    t.g0[k] = (float)rec_lo[k];
    t.g1[k] = (float)rec_hi[k];
  }
  for (int k = 0; k < L; k++) {
    h->ana.a[k] = t.h0[k];
    h->ana.b[k] = t.h1[k];
    h->syn.a[k] = t.g0[k];
    h->syn.b[k] = t.g1[k];
  }
  if (cudaMalloc(&h->taps, sizeof(Taps)) != cudaSuccess)
    return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  if (cudaMemcpy(h->taps, &t, sizeof(Taps), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(TCB_ERR_CUDA, "cudaMemcpy failed");
  size_t maxband = 0, maxtmp = 0;
  for (int k = 0; k < level; k++) {
    int Ho = h->H[k + 1], Wo = h->W[k + 1];
    float *y = nullptr;
    if (cudaMalloc(&y, (size_t)nz * 4 * Ho * Wo * sizeof(float)) != cudaSuccess)
      return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    h->Y.push_back(y);
    // damping factors (remove_stripe.py:270-274), 1/Ho of the inverse FFT folded in
    int nc = Ho / 2 + 1;
    std::vector<double> yh(Ho);
    for (int q = 0; q < Ho; q++) yh[q] = ((-Ho + 2 * q) + 1) / 2.0;
    std::vector<float> d(nc);
    for (int q = 0; q < nc; q++) {
      double v = yh[(q + Ho / 2) % Ho];  // ifftshift, first nc entries
      d[q] = (float)(-std::expm1(-v * v / (2.0 * (double)sigma * sigma)) / Ho);
    }
    float *dd = nullptr;
    if (cudaMalloc(&dd, nc * sizeof(float)) != cudaSuccess)
      return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    h->damp.push_back(dd);
    if (cudaMemcpy(dd, d.data(), nc * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(TCB_ERR_CUDA, "cudaMemcpy failed");
    cufftHandle p1 = 0, p2 = 0;
    int len[1] = {Ho};
    int batch = (int)(nz * Wo);
    if (cufftPlanMany(&p1, 1, len, nullptr, 1, Ho, nullptr, 1, nc, CUFFT_R2C, batch) !=
            CUFFT_SUCCESS ||
        cufftPlanMany(&p2, 1, len, nullptr, 1, nc, nullptr, 1, Ho, CUFFT_C2R, batch) !=
            CUFFT_SUCCESS)
      return fail(TCB_ERR_CUFFT, "cufftPlanMany failed");
    h->r2c.push_back(p1);
    h->c2r.push_back(p2);
    // the direct damping: modes k with g_k above 1e-12, padded to 8, 16 or 32
    // (the extra ones carry their exact, negligible weights); the mode and its
    // mirror H - k must be distinct
    int need = 0;
    while (need < Ho) {
      const double v = (Ho % 2) ? (double)need : need + 0.5;
      if (std::exp(-v * v / (2.0 * (double)sigma * sigma)) < 1e-12) break;
      need++;
    }
    int V1 = need <= 8 ? 8 : need <= 16 ? 16 : need <= 32 ? 32 : 0;
    if (2 * V1 >= Ho || std::getenv("TCB_FW_DAMP") != nullptr) V1 = 0;
    float2 *mc = nullptr;
    float *mg = nullptr;
    if (V1) {
      std::vector<float2> tab((size_t)V1 * Ho);
      std::vector<float> wt(V1);
      for (int k = 0; k < V1; k++) {
        for (int q = 0; q < Ho; q++) {
          // 2 pi k q / H reduced exactly: (k q mod H) / H
          const double a = 2.0 * M_PI * (double)(((long long)k * q) % Ho) / (double)Ho;
          tab[(size_t)k * Ho + q] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        const double v = (Ho % 2) ? (double)k : k + 0.5;
        const double g = std::exp(-v * v / (2.0 * (double)sigma * sigma)) / Ho;
        // bin 0 is its own mirror; bin k >= 1 comes with bin H - k, whose
        // factor the half-spectrum inverse takes from bin k
        wt[k] = (float)(k == 0 ? g : 2.0 * g);
      }
      if (cudaMalloc(&mc, tab.size() * sizeof(float2)) != cudaSuccess ||
          cudaMalloc(&mg, V1 * sizeof(float)) != cudaSuccess) {
        cudaFree(mc);
        return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
      }
      if (cudaMemcpy(mc, tab.data(), tab.size() * sizeof(float2), cudaMemcpyHostToDevice) !=
              cudaSuccess ||
          cudaMemcpy(mg, wt.data(), V1 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(mc);
        cudaFree(mg);
        return fail(TCB_ERR_CUDA, "cudaMemcpy failed");
      }
    }
    h->modes.push_back(V1);
    h->mcs.push_back(mc);
    h->mgw.push_back(mg);
    maxband = std::max(maxband, (size_t)nz * Ho * Wo);
    maxtmp = std::max(maxtmp, (size_t)nz * 2 * h->H[k] * Wo);          // afb rows output
    maxtmp = std::max(maxtmp, (size_t)nz * 2 * (2 * Ho - L + 2) * Wo);  // sfb cols output
  }
  if (cudaMalloc(&h->tmp, maxtmp * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->bt, maxband * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->spec, (maxband / 2 + (size_t)nz * h->W[1] + 16) * sizeof(float2)) !=
          cudaSuccess)
    return fail(TCB_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  h->tmp_elems = maxtmp;
  *out = h;
  return TCB_OK;
}

// Ring removal in place on padded sinograms sino [nz][nproj_pad][ni] (slice
// stride sstride elements): rows [(pad)/2, (pad)/2 + nproj) hold the data,
// the other rows must be zero on entry (they are overwritten).
extern "C" int tcb_stripe_fw_apply_sino(tcb_stripe_fw *h, float *sino, size_t sstride,
                                        void *stream) {
  TCB_CHECK_ARG(h && h->taps, "tcb_stripe_fw_apply_sino: null or freed handle");
  TCB_CHECK_ARG(sino, "tcb_stripe_fw_apply_sino: null pointer");
  TCB_CHECK_ARG(sstride >= (size_t)h->nproj_pad * h->ni, "tcb_stripe_fw_apply_sino: stride");
  cudaStream_t s = (cudaStream_t)stream;
  const int B = h->nz, L = h->L;
  // forward
  for (int k = 0; k < h->level; k++) {
    int Hk = h->H[k], Wk = h->W[k], Ho = h->H[k + 1], Wo = h->W[k + 1];
    const float *x;
    long long xsz;
    int xsx;
    if (k == 0) {
      x = sino;
      xsz = (long long)sstride;
      xsx = Wk;
    } else {
      x = h->Y[k - 1];  // LL channel of the previous level
      xsz = 4LL * Hk * Wk;
      xsx = Wk;
    }
    int pw = 2 * (Wo - 1) - Wk + L, ph = 2 * (Ho - 1) - Hk + L;
    long long n1 = (long long)B * Hk * Wo;
    {
      StageTimer st("fw_afb_rows", s);
      switch (blocked_length(L) ? L : 0) {
        case 2: launch_afb_rows<2>(h, x, xsz, xsx, B, Hk, Wk, Wo, pw / 2, s); break;
        case 10: launch_afb_rows<10>(h, x, xsz, xsx, B, Hk, Wk, Wo, pw / 2, s); break;
        case 32: launch_afb_rows<32>(h, x, xsz, xsx, B, Hk, Wk, Wo, pw / 2, s); break;
        default:
          afb_rows<<<ceil_div(n1, 256), 256, 0, s>>>(x, xsz, xsx, h->tmp, B, Hk, Wk, Wo, pw / 2,
                                                     h->taps);
      }
    }
    TCB_LAUNCH_CHECK();
    long long n2 = (long long)B * 2 * Ho * Wo;
    {
      StageTimer st("fw_afb_cols", s);
      switch (blocked_length(L) ? L : 0) {
        case 2: launch_afb_cols<2>(h, h->Y[k], B, Hk, Wo, Ho, ph / 2, s); break;
        case 10: launch_afb_cols<10>(h, h->Y[k], B, Hk, Wo, Ho, ph / 2, s); break;
        case 32: launch_afb_cols<32>(h, h->Y[k], B, Hk, Wo, Ho, ph / 2, s); break;
        default:
          afb_cols<<<ceil_div(n2, 256), 256, 0, s>>>(h->tmp, h->Y[k], B, Hk, Wo, Ho, ph / 2,
                                                     h->taps);
      }
    }
    TCB_LAUNCH_CHECK();
    StageTimer std_("fw_damp", s);
    // damp band 1 (index 2 of the level: high-pass along the detector, low-pass along angles)
    float *band = h->Y[k] + 2LL * Ho * Wo;
    if (h->modes[k]) {
      const dim3 gd(ceil_div(Wo, 32), B), bd(32, DM_R);
      switch (h->modes[k]) {
        case 8: damp_modes<8><<<gd, bd, 0, s>>>(band, 4LL * Ho * Wo, Ho, Wo, h->mcs[k], h->mgw[k]); break;
        case 16: damp_modes<16><<<gd, bd, 0, s>>>(band, 4LL * Ho * Wo, Ho, Wo, h->mcs[k], h->mgw[k]); break;
        default: damp_modes<32><<<gd, bd, 0, s>>>(band, 4LL * Ho * Wo, Ho, Wo, h->mcs[k], h->mgw[k]);
      }
      TCB_LAUNCH_CHECK();
      count_launch();
      continue;
    }
    dim3 tb(32, 8);
    dim3 g1(ceil_div(Wo, 32), ceil_div(Ho, 32), B);
    transpose_bands<<<g1, tb, 0, s>>>(band, 4LL * Ho * Wo, h->bt, (long long)Ho * Wo, Ho, Wo);
    TCB_LAUNCH_CHECK();
    TCB_CUFFT(cufftSetStream(h->r2c[k], s));
    TCB_CUFFT(cufftSetStream(h->c2r[k], s));
    TCB_CUFFT(cufftExecR2C(h->r2c[k], h->bt, (cufftComplex *)h->spec));
    int nc = Ho / 2 + 1;
    long long tot = (long long)B * Wo * nc;
    damp_kernel<<<ceil_div(tot, 256), 256, 0, s>>>(h->spec, h->damp[k], nc, tot);
    TCB_LAUNCH_CHECK();
    TCB_CUFFT(cufftExecC2R(h->c2r[k], (cufftComplex *)h->spec, h->bt));
    dim3 g2(ceil_div(Ho, 32), ceil_div(Wo, 32), B);
    transpose_bands<<<g2, tb, 0, s>>>(h->bt, (long long)Ho * Wo, band, 4LL * Ho * Wo, Wo, Ho);
    TCB_LAUNCH_CHECK();
    count_launch(5);
  }
  // inverse
  for (int k = h->level - 1; k >= 0; k--) {
    int Hi = h->H[k + 1], Wi = h->W[k + 1];
    int Hc = 2 * Hi - L + 2;  // rows after the column synthesis
    long long n1 = (long long)B * 2 * Hc * Wi;
    {
      StageTimer st("fw_sfb_cols", s);
      switch (blocked_length(L) ? L : 0) {
        case 2: launch_sfb_cols<2>(h, h->Y[k], Hi, Wi, B, Hc, s); break;
        case 10: launch_sfb_cols<10>(h, h->Y[k], Hi, Wi, B, Hc, s); break;
        case 32: launch_sfb_cols<32>(h, h->Y[k], Hi, Wi, B, Hc, s); break;
        default:
          sfb_cols<<<ceil_div(n1, 256), 256, 0, s>>>(h->Y[k], 4LL * Hi * Wi, Hi, Wi, Wi, h->tmp,
                                                     B, Hc, h->taps);
      }
    }
    TCB_LAUNCH_CHECK();
    // reconstruction of level k's input, cropped to its size, into the LL
    // channel of the level above (or into the sinograms)
    int Hd = h->H[k], Wd = h->W[k];
    float *dst;
    long long dsz;
    if (k == 0) {
      dst = sino;
      dsz = (long long)sstride;
    } else {
      dst = h->Y[k - 1];
      dsz = 4LL * Hd * Wd;
    }
    int Hrows = std::min(Hd, Hc);
    long long n2 = (long long)B * Hrows * Wd;
    StageTimer st("fw_sfb_rows", s);
    switch (blocked_length(L) ? L : 0) {
      case 2: launch_sfb_rows<2>(h, Hc, Wi, dst, dsz, Wd, Hrows, B, s); break;
      case 10: launch_sfb_rows<10>(h, Hc, Wi, dst, dsz, Wd, Hrows, B, s); break;
      case 32: launch_sfb_rows<32>(h, Hc, Wi, dst, dsz, Wd, Hrows, B, s); break;
      default:
        sfb_rows<<<ceil_div(n2, 256), 256, 0, s>>>(h->tmp, Hc, Wi, dst, dsz, Wd, Hrows, Wd, B,
                                                   h->taps);
    }
    TCB_LAUNCH_CHECK();
    count_launch(2);
  }
  return TCB_OK;
}

extern "C" int tcb_stripe_fw_destroy(tcb_stripe_fw *h) {
  if (!h) return TCB_OK;
  fw_release(h);
  delete h;
  return TCB_OK;
}
