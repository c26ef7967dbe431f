// Inverse (exponent +i) complex FFTs of power-of-two length N in shared
// memory, one transform per group of T = N/16 threads, each thread holding
// 16 values in registers between stages.
//
// Algorithm: Stockham autosort, decimation in time (the formulation of
// Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC 2008): stage s with radix R and current
// sub-length Ns takes butterfly b from elements b + r*N/R (r < R),
// multiplies element r by w^(r*(b mod Ns)) with w = exp(2*pi*i/(Ns*R)),
// applies the R-point DFT and stores output r at
// (b/Ns)*Ns*R + (b mod Ns) + r*Ns.  After the last stage the data is in
// natural order.  Radix-16 stages (a 4 x 4 register DFT) come first, then
// one radix-2/4/8 stage when N is not a power of 16.
//
// Unnormalised, like cuFFT's CUFFT_INVERSE.  The twiddles come from a
// per-stage table computed in float64 on the host (twiddle_table below):
// stage S keeps w^(2^j * k) for j < log2(R), k in [0, Ns) at
// tw[offset(S) + j*Ns + k], so the lanes of a warp, which hold consecutive
// k, read consecutive entries; w^(r*k) is the product of the entries of the
// set bits of r (at most 3 roundings for r < 16).  log2(R) loads instead of
// R - 1 keep the tables of all stages small enough to stay in L1 next to
// the data streams.  The first stage
// reads its inputs through a caller functor (global memory), the last stage
// hands its outputs to another functor (global memory, with any pruning or
// epilogue the caller wants); the stages in between go through shared
// memory with one padding slot every 16 elements.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

namespace tcb {
namespace fftk {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 mul_i(float2 a) { return make_float2(-a.y, a.x); }

// exp(2*pi*i*m/16) for the 4 x 4 decomposition (cos/sin of multiples of pi/8)
constexpr float C8 = 0.923879532511286756f;   // cos(pi/8)
constexpr float S8 = 0.382683432365089772f;   // sin(pi/8)
constexpr float R2 = 0.707106781186547524f;   // cos(pi/4)

__device__ __forceinline__ void dft2(float2 &a, float2 &b) {
  float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
  float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
  float2 s13 = cadd(a1, a3), d13 = mul_i(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}

// v[0..7] -> inverse 8-point DFT in natural order (2 x 4 split)
__device__ __forceinline__ void dft8(float2 *v) {
  float2 a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
  float2 b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
  dft4(a0, a1, a2, a3);
  dft4(b0, b1, b2, b3);
  b1 = cmul(b1, make_float2(R2, R2));
  b2 = mul_i(b2);
  b3 = cmul(b3, make_float2(-R2, R2));
  v[0] = cadd(a0, b0); v[4] = csub(a0, b0);
  v[1] = cadd(a1, b1); v[5] = csub(a1, b1);
  v[2] = cadd(a2, b2); v[6] = csub(a2, b2);
  v[3] = cadd(a3, b3); v[7] = csub(a3, b3);
}

// v[0..15] -> inverse 16-point DFT in natural order (4 x 4 split)
__device__ __forceinline__ void dft16(float2 *v) {
  float2 b[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
    b[n2][0] = v[n2];
    b[n2][1] = v[4 + n2];
    b[n2][2] = v[8 + n2];
    b[n2][3] = v[12 + n2];
    dft4(b[n2][0], b[n2][1], b[n2][2], b[n2][3]);
  }
  // twiddles exp(2*pi*i*n2*k1/16)
  b[1][1] = cmul(b[1][1], make_float2(C8, S8));
  b[1][2] = cmul(b[1][2], make_float2(R2, R2));
  b[1][3] = cmul(b[1][3], make_float2(S8, C8));
  b[2][1] = cmul(b[2][1], make_float2(R2, R2));
  b[2][2] = mul_i(b[2][2]);
  b[2][3] = cmul(b[2][3], make_float2(-R2, R2));
  b[3][1] = cmul(b[3][1], make_float2(S8, C8));
  b[3][2] = cmul(b[3][2], make_float2(-R2, R2));
  b[3][3] = cmul(b[3][3], make_float2(-C8, -S8));
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    float2 c0 = b[0][k1], c1 = b[1][k1], c2 = b[2][k1], c3 = b[3][k1];
    dft4(c0, c1, c2, c3);
    v[k1] = c0;
    v[k1 + 4] = c1;
    v[k1 + 8] = c2;
    v[k1 + 12] = c3;
  }
}

template <int R> __device__ __forceinline__ void dft(float2 *v) {
  if constexpr (R == 16) dft16(v);
  else if constexpr (R == 8) dft8(v);
  else if constexpr (R == 4) dft4(v[0], v[1], v[2], v[3]);
  else dft2(v[0], v[1]);
}

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
template <int N> struct Plan {
  static_assert(N >= 256 && N <= 8192 && (N & (N - 1)) == 0, "N: power of two in [256, 8192]");
  static constexpr int NS16 = ilog2(N) / 4;                    // radix-16 stages
  static constexpr int RL = N >> (4 * NS16);                   // last radix (1 = none)
  static constexpr int NST = NS16 + (RL > 1 ? 1 : 0);
  static constexpr int T = N / 16;                             // threads per transform
  static constexpr int PADDED = N + N / 16;                    // smem slots per transform
};
template <int N, int S> constexpr int radix_of() {
  return S < Plan<N>::NS16 ? 16 : Plan<N>::RL;
}
template <int N, int S> constexpr int ns_of() {
  if constexpr (S == 0) return 1;
  else return ns_of<N, S - 1>() * radix_of<N, S - 1>();
}

// First twiddle of stage S in the per-stage table (stage 0 needs none).
template <int N, int S> constexpr int tw_offset() {
  if constexpr (S <= 1) return 0;
  else return tw_offset<N, S - 1>() + ilog2(radix_of<N, S - 1>()) * ns_of<N, S - 1>();
}

// w^(r*k) for r in [1, R) from the log2(R) table entries w^(2^j * k).
template <int R>
__device__ __forceinline__ void stage_twiddles(const float2 *__restrict__ t, int ns, int k,
                                               float2 (&w)[16]) {
  w[1] = __ldg(t + k);
  if constexpr (R >= 4) {
    w[2] = __ldg(t + ns + k);
    w[3] = cmul(w[1], w[2]);
  }
  if constexpr (R >= 8) {
    w[4] = __ldg(t + 2 * ns + k);
    w[5] = cmul(w[1], w[4]);
    w[6] = cmul(w[2], w[4]);
    w[7] = cmul(w[3], w[4]);
  }
  if constexpr (R >= 16) {
    w[8] = __ldg(t + 3 * ns + k);
#pragma unroll
    for (int r = 1; r < 8; r++) w[8 + r] = cmul(w[r], w[8]);
  }
}

__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

// One stage (and, recursively, the ones after it).  sm: this transform's
// padded shared buffer; tid in [0, T); in(e) -> float2 for stage 0;
// out(o, value) for the last stage.  SYNC_OUT: a block barrier between the
// last stage's shared reads and the out calls, so out may write sm.  Threads
// with active == false only take part in the barriers.
template <int N, int S, bool SYNC_OUT, class In, class Out>
__device__ __forceinline__ void run_stage(float2 (&v)[16], float2 *sm, int tid,
                                          const float2 *__restrict__ tw, In &in, Out &out,
                                          bool active) {
  constexpr int R = radix_of<N, S>(), Ns = ns_of<N, S>(), NB = 16 / R;
  constexpr int T = Plan<N>::T;
  if (active) {
#pragma unroll
    for (int q = 0; q < NB; q++) {
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int e = tid + q * T + r * (N / R);
        if constexpr (S == 0) v[q * R + r] = in(e);
        else v[q * R + r] = sm[pad16(e)];
      }
    }
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = tid + q * T;
      if constexpr (Ns > 1) {
        const int k = b & (Ns - 1);
        float2 w[16];
        stage_twiddles<R>(tw + tw_offset<N, S>(), Ns, k, w);
#pragma unroll
        for (int r = 1; r < R; r++) v[q * R + r] = cmul(v[q * R + r], w[r]);
      }
      dft<R>(&v[q * R]);
    }
  }
  if constexpr (S == Plan<N>::NST - 1) {
    if constexpr (SYNC_OUT) __syncthreads();
    if (active) {
#pragma unroll
      for (int q = 0; q < NB; q++)
#pragma unroll
        for (int r = 0; r < R; r++) out(tid + q * T + r * Ns, v[q * R + r]);
    }
  } else {
    __syncthreads();
    if (active) {
#pragma unroll
      for (int q = 0; q < NB; q++) {
        const int b = tid + q * T;
        const int base = (b / Ns) * Ns * R + (b & (Ns - 1));
#pragma unroll
        for (int r = 0; r < R; r++) sm[pad16(base + r * Ns)] = v[q * R + r];
      }
    }
    __syncthreads();
    run_stage<N, S + 1, SYNC_OUT>(v, sm, tid, tw, in, out, active);
  }
}

// Inverse FFT of one length-N transform by its T = N/16 threads.  Every
// thread of the block must call it the same number of times (it contains
// __syncthreads); the caller's block may hold several transforms side by
// side, each with its own sm buffer of Plan<N>::PADDED slots, or run a
// transform on part of its threads (active false on the others).
template <int N, bool SYNC_OUT = false, class In, class Out>
__device__ __forceinline__ void ifft(float2 *sm, int tid, const float2 *__restrict__ tw, In in,
                                     Out out, bool active = true) {
  float2 v[16];
  run_stage<N, 0, SYNC_OUT>(v, sm, tid, tw, in, out, active);
}

// Host: the per-stage twiddle table of a length-n transform (n a power of
// two in [256, 8192]), entries exp(2*pi*i*2^j*k/(Ns*R)) in float64 rounded
// to float, in the order run_stage reads them.
inline std::vector<float2> twiddle_table(int n) {
  int ns16 = 0;
  while ((16 << (4 * ns16)) <= n) ns16++;
  const int rl = n >> (4 * ns16);
  const int nst = ns16 + (rl > 1 ? 1 : 0);
  std::vector<float2> t;
  int ns = 1;
  for (int s = 0; s < nst; s++) {
    const int r_s = s < ns16 ? 16 : rl;
    if (s > 0)
      for (int p = 1; p < r_s; p *= 2)
        for (int k = 0; k < ns; k++) {
          const double a = 2.0 * M_PI * (double)p * (double)k / ((double)ns * r_s);
          t.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
    ns *= r_s;
  }
  return t;
}

}  // namespace fftk
}  // namespace tcb
