// Fused fp32 FBP filter: edge padding, the spectral filter with the centre
// phase ramp, the crop and (optionally) FourierRec's projection FFT, in one
// kernel per pair of sinogram rows.
//
// The reference filters a row of n samples by edge-padding it to ne = 4n,
// R2C, multiplying by w = wfilter * exp(-2 pi i (-center + sht + n/2) t),
// C2R and cropping n samples (src/tomocupy/reconstruction/backproj_functions.py:93-109,
// src/cuda/cfunc_filter.cu:49-61, src/include/kernels_filter.cuh:4-18).
// The chain is linear: y[j] = sum_i T[j][i] x[i] with
// T[j][i] = hz[(j - i) mod ne] (hz = C2R(w), unnormalised) except in
// columns 0 and n-1, which also collect the edge padding.  So
//
//   y = x (*) h_L  +  x[0] * A  +  x[n-1] * B
//
// where (*) is a circular convolution of length L >= 2n (a power of two)
// with h_L[m] = hz[m] for m < n, hz[m - L + ne] for m > L - n, 0 between
// (indices j - i lie in (-n, n), so nothing wraps), and
// A[j] = T[j][0] - hz[j], B[j] = T[j][n-1] - hz[(j - n + 1) mod ne] are the
// folded padding columns.  The convolution runs as two length-L FFTs in
// shared memory instead of cuFFT's three passes at length 4n through HBM.
//
// Two slices go through one complex transform (slice q real, slice q + half
// imaginary: the packing of FourierRec.backprojection,
// src/tomocupy/reconstruction/fourierrec.py:63-68).  Their kernels may
// differ (centre sweeps): with X = DFT(x_a + i x_b),
// Y[k] = (X[k] + conj X[-k])/2 * H_a[k] + (X[k] - conj X[-k])/2 * H_b[k]
// is the spectrum of y_a + i y_b.  Output modes: the filtered real rows,
// the packed complex rows, or (n a power of two) the packed rows' forward
// DFT of length n, which is what FourierRec's projection FFT
// (cfunc_fourierrec.cu:67-94, the 1D FFT before the gridding) would make.
//
// H = DFT_L(h_L)/L and A, B are computed on the host in float64 from hz.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <vector>

#include "common.cuh"
#include "fft_pow2.cuh"

struct tcb_fftfilter {
  size_t nproj = 0, nz = 0, n = 0, nkern = 0;
  int L = 0;               // convolution length: next power of two >= 2n
  bool spectrum_ok = false;  // n a power of two in [256, 4096]
  float2 *H = nullptr;     // [nkern][L] DFT_L(h_L) / L
  float2 *AB = nullptr;    // [nkern][n] folded padding columns (A[j], B[j])
  float2 *twL = nullptr;   // per-stage twiddles of length L
  float2 *twn = nullptr;   // per-stage twiddles of length n (spectrum mode)
  bool ready = false;
};

namespace tcb {
namespace fff {

enum { OUT_ROWS = TCB_FFF_OUT_ROWS, OUT_PAIRS = TCB_FFF_OUT_PAIRS,
       OUT_SPECTRUM = TCB_FFF_OUT_SPECTRUM };

struct Args {
  const float *x;
  size_t ldx, xoff;
  int nproj, nz, half, n;
  int shared_kern, kern0;
  const float2 *H;
  const float2 *AB;
  const float2 *twL, *twn;
  void *out;
  size_t ldo;
};

using fftk::cmul;
using fftk::pad16;

// One block per (slice pair q, angle p); L/16 threads.
template <int L, int MODE>
__global__ void __launch_bounds__(L / 16, (16384 / L < 16 ? 16384 / L : 16))
    fff_kernel(const Args a) {
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int p = (int)(blockIdx.x % (unsigned)a.nproj);
  const int q = (int)(blockIdx.x / (unsigned)a.nproj);
  const int n = a.n;
  const int zb = q + a.half;
  const bool hasb = zb < a.nz;
  const float *xa = a.x + ((size_t)q * a.nproj + p) * a.ldx + a.xoff;
  const float *xb = hasb ? a.x + ((size_t)zb * a.nproj + p) * a.ldx + a.xoff : xa;
  const int ka = a.shared_kern ? 0 : a.kern0 + q;
  const int kb = (a.shared_kern || !hasb) ? ka : a.kern0 + zb;

  // 1) R = IDFT_L(conj(x_a + i x_b)), zero padded; DFT(x) = conj(R)
  fftk::ifft<L, true>(
      sm, tid, a.twL,
      [&](int e) {
        if (e < n) return make_float2(__ldg(xa + e), hasb ? -__ldg(xb + e) : 0.f);
        return make_float2(0.f, 0.f);
      },
      [&](int o, float2 v) { sm[pad16(o)] = v; });
  __syncthreads();

  // 2) y = IDFT_L(Y) (1/L folded into H), then the padding columns
  const float2 *Ha = a.H + (size_t)ka * L, *Hb = a.H + (size_t)kb * L;
  const float2 *ABa = a.AB + (size_t)ka * n, *ABb = a.AB + (size_t)kb * n;
  const float xa0 = __ldg(xa), xan = __ldg(xa + n - 1);
  const float xb0 = hasb ? __ldg(xb) : 0.f, xbn = hasb ? __ldg(xb + n - 1) : 0.f;
  const bool same = ka == kb;
  const size_t row = (size_t)q * a.nproj + p;
  auto in2 = [&](int e) {
    const float2 r = sm[pad16(e)];
    const float2 X = make_float2(r.x, -r.y);
    if (same) return cmul(X, __ldg(Ha + e));
    const float2 rm = sm[pad16((L - e) & (L - 1))];  // conj X[-e]
    const float2 P = make_float2(0.5f * (X.x + rm.x), 0.5f * (X.y + rm.y));
    const float2 Q = make_float2(0.5f * (X.x - rm.x), 0.5f * (X.y - rm.y));
    const float2 u = cmul(P, __ldg(Ha + e)), w = cmul(Q, __ldg(Hb + e));
    return make_float2(u.x + w.x, u.y + w.y);
  };
  auto fix = [&](int o, float2 v) {
    const float2 ca = __ldg(ABa + o);
    const float2 cb = same ? ca : __ldg(ABb + o);
    v.x += xa0 * ca.x + xan * ca.y;
    v.y += xb0 * cb.x + xbn * cb.y;
    return v;
  };
  if constexpr (MODE == OUT_ROWS) {
    float *oa = (float *)a.out + row * a.ldo;
    float *ob = hasb ? (float *)a.out + ((size_t)zb * a.nproj + p) * a.ldo : oa;
    fftk::ifft<L, false>(sm, tid, a.twL, in2, [&](int o, float2 v) {
      if (o < n) {
        v = fix(o, v);
        oa[o] = v.x;
        if (hasb) ob[o] = v.y;
      }
    });
  } else if constexpr (MODE == OUT_PAIRS) {
    float2 *oc = (float2 *)a.out + row * n;
    fftk::ifft<L, false>(sm, tid, a.twL, in2, [&](int o, float2 v) {
      if (o < n) oc[o] = fix(o, v);
    });
  } else {
    fftk::ifft<L, true>(sm, tid, a.twL, in2, [&](int o, float2 v) {
      if (o < n) sm[pad16(o)] = fix(o, v);
    });
    __syncthreads();
    // 3) forward DFT_n of the packed row: conj(IDFT_n(conj(y)))
    constexpr int N1 = L / 2;
    float2 *oc = (float2 *)a.out + row * N1;
    fftk::ifft<N1, false>(
        sm, tid, a.twn,
        [&](int e) {
          const float2 v = sm[pad16(e)];
          return make_float2(v.x, -v.y);
        },
        [&](int o, float2 v) { oc[o] = make_float2(v.x, -v.y); }, tid < N1 / 16);
  }
}

// Host float64 FFT (iterative radix-2, forward e^{-i}), for the kernel spectra.
void fft64(std::vector<std::complex<double>> &v) {
  const size_t N = v.size();
  for (size_t i = 1, j = 0; i < N; i++) {
    size_t bit = N >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(v[i], v[j]);
  }
  for (size_t len = 2; len <= N; len <<= 1) {
    const double ang = -2.0 * M_PI / (double)len;
    for (size_t i = 0; i < N; i += len)
      for (size_t k = 0; k < len / 2; k++) {
        const std::complex<double> w(std::cos(ang * (double)k), std::sin(ang * (double)k));
        const std::complex<double> u = v[i + k], t = v[i + k + len / 2] * w;
        v[i + k] = u + t;
        v[i + k + len / 2] = u - t;
      }
  }
}

template <int L>
cudaError_t set_attrs() {
  const int smem = (int)(fftk::Plan<L>::PADDED * sizeof(float2));
  cudaError_t e = cudaFuncSetAttribute(fff_kernel<L, OUT_ROWS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fff_kernel<L, OUT_PAIRS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if constexpr (L >= 512) {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(fff_kernel<L, OUT_SPECTRUM>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  }
  return e;
}

template <int L>
void launch(const Args &a, int mode, unsigned blocks, cudaStream_t s) {
  const size_t smem = fftk::Plan<L>::PADDED * sizeof(float2);
  if (mode == OUT_ROWS)
    fff_kernel<L, OUT_ROWS><<<blocks, L / 16, smem, s>>>(a);
  else if (mode == OUT_PAIRS)
    fff_kernel<L, OUT_PAIRS><<<blocks, L / 16, smem, s>>>(a);
  else if constexpr (L >= 512)
    fff_kernel<L, OUT_SPECTRUM><<<blocks, L / 16, smem, s>>>(a);
}

void release(tcb_fftfilter *h) {
  cudaFree(h->H);
  cudaFree(h->AB);
  cudaFree(h->twL);
  cudaFree(h->twn);
  h->H = h->twL = h->twn = nullptr;
  h->AB = nullptr;
}

}  // namespace fff
}  // namespace tcb

using namespace tcb;
using namespace tcb::fff;

extern "C" int tcb_fftfilter_create(tcb_fftfilter **out, size_t nproj, size_t nz, size_t n,
                                    size_t nkern) {
  TCB_CHECK_ARG(out, "tcb_fftfilter_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 1 && nz >= 1 && nkern >= 1, "tcb_fftfilter_create: empty sizes");
  TCB_CHECK_ARG(n >= 2 && n <= 4096, "tcb_fftfilter_create: n must be in [2, 4096]");
  TCB_CHECK_ARG(nproj * nz < (1ull << 31) && nkern <= 65536,
                "tcb_fftfilter_create: sizes too large");
  int L = 256;
  while ((size_t)L < 2 * n) L *= 2;
  auto *h = new tcb_fftfilter{};
  h->nproj = nproj;
  h->nz = nz;
  h->n = n;
  h->nkern = nkern;
  h->L = L;
  h->spectrum_ok = n >= 256 && (n & (n - 1)) == 0 && (size_t)L == 2 * n;
  const std::vector<float2> twL = fftk::twiddle_table(L);
  std::vector<float2> twn;
  if (h->spectrum_ok) twn = fftk::twiddle_table((int)n);
  cudaError_t e = cudaSuccess;
  if (cudaMalloc(&h->H, nkern * (size_t)L * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&h->AB, nkern * n * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&h->twL, twL.size() * sizeof(float2)) != cudaSuccess ||
      (h->spectrum_ok && cudaMalloc(&h->twn, twn.size() * sizeof(float2)) != cudaSuccess)) {
    cudaGetLastError();
    release(h);
    delete h;
    set_error("tcb_fftfilter_create: out of device memory");
    return TCB_ERR_OUT_OF_MEMORY;
  }
  e = cudaMemcpy(h->twL, twL.data(), twL.size() * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && h->spectrum_ok)
    e = cudaMemcpy(h->twn, twn.data(), twn.size() * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    switch (L) {
      case 256: e = set_attrs<256>(); break;
      case 512: e = set_attrs<512>(); break;
      case 1024: e = set_attrs<1024>(); break;
      case 2048: e = set_attrs<2048>(); break;
      case 4096: e = set_attrs<4096>(); break;
      default: e = set_attrs<8192>(); break;
    }
  }
  if (e != cudaSuccess) {
    release(h);
    delete h;
    set_error("tcb_fftfilter_create: %s", cudaGetErrorString(e));
    return TCB_ERR_CUDA;
  }
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_fftfilter_set_kernels(tcb_fftfilter *h, const double *hz, size_t ne,
                                         size_t pad, void *stream) {
  TCB_CHECK_ARG(h && hz, "tcb_fftfilter_set_kernels: null pointer");
  TCB_CHECK_ARG(h->H, "tcb_fftfilter_set_kernels: handle was freed");
  const size_t n = h->n, nk = h->nkern, L = (size_t)h->L;
  TCB_CHECK_ARG(ne >= n && pad + n <= ne, "tcb_fftfilter_set_kernels: need pad + n <= ne");
  TCB_CHECK_ARG(ne < (1u << 30), "tcb_fftfilter_set_kernels: ne too large");
  std::vector<float2> Hh(nk * L);
  std::vector<float2> ABh(nk * n);
  std::vector<double> cs(2 * ne + 1);
  std::vector<std::complex<double>> v(L);
  for (size_t k = 0; k < nk; k++) {
    const double *hk = hz + k * ne;
    for (size_t d = 0; d < ne; d++)
      if (!std::isfinite(hk[d])) {
        set_error("tcb_fftfilter_set_kernels: non-finite kernel value");
        return TCB_ERR_INVALID_ARGUMENT;
      }
    // h_L: offsets 0..n-1 at the front, -(n-1)..-1 at the back
    std::fill(v.begin(), v.end(), std::complex<double>(0.0, 0.0));
    for (size_t m = 0; m < n; m++) v[m] = hk[m];
    for (size_t d = 1; d < n; d++) v[L - d] = hk[ne - d];
    fft64(v);
    for (size_t m = 0; m < L; m++)
      Hh[k * L + m] = make_float2((float)(v[m].real() / (double)L),
                                  (float)(v[m].imag() / (double)L));
    // folded padding columns by prefix sums over two periods:
    // cs[t] = sum_{u=-ne}^{t-ne-1} hk[u mod ne]
    cs[0] = 0.0;
    for (size_t t = 0; t < 2 * ne; t++) cs[t + 1] = cs[t] + hk[t % ne];
    auto S = [&](long long a, long long b) {  // sum_{d=a}^{b} hk[d mod ne], -ne <= a
      return cs[(size_t)(b + 1 + (long long)ne)] - cs[(size_t)(a + (long long)ne)];
    };
    for (size_t j = 0; j < n; j++) {
      const double col0 = S((long long)j, (long long)(j + pad));
      const double coln = S((long long)j + (long long)pad - (long long)ne + 1,
                            (long long)j - (long long)n + 1);
      ABh[k * n + j] = make_float2((float)(col0 - hk[j % ne]),
                                   (float)(coln - hk[(j + ne - (n - 1)) % ne]));
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  TCB_CUDA(cudaMemcpyAsync(h->H, Hh.data(), Hh.size() * sizeof(float2), cudaMemcpyHostToDevice,
                           s));
  TCB_CUDA(cudaMemcpyAsync(h->AB, ABh.data(), ABh.size() * sizeof(float2),
                           cudaMemcpyHostToDevice, s));
  TCB_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  h->ready = true;
  return TCB_OK;
}

extern "C" int tcb_fftfilter_apply(tcb_fftfilter *h, const float *x, size_t ldx, size_t xoff,
                                   size_t nz, size_t kern0, void *out, int out_mode, size_t ldo,
                                   void *stream) {
  TCB_CHECK_ARG(h && x && out, "tcb_fftfilter_apply: null pointer");
  TCB_CHECK_ARG(h->H, "tcb_fftfilter_apply: handle was freed");
  TCB_CHECK_ARG(h->ready, "tcb_fftfilter_apply: tcb_fftfilter_set_kernels was not called");
  TCB_CHECK_ARG(nz >= 1 && nz <= h->nz, "tcb_fftfilter_apply: nz out of range");
  TCB_CHECK_ARG(ldx >= xoff + h->n, "tcb_fftfilter_apply: ldx < xoff + n");
  TCB_CHECK_ARG(out_mode == OUT_ROWS || out_mode == OUT_PAIRS || out_mode == OUT_SPECTRUM,
                "tcb_fftfilter_apply: unknown out_mode %d", out_mode);
  TCB_CHECK_ARG(out_mode != OUT_ROWS || ldo >= h->n, "tcb_fftfilter_apply: ldo < n");
  TCB_CHECK_ARG(out_mode == OUT_ROWS || nz % 2 == 0,
                "tcb_fftfilter_apply: paired output needs an even slice count");
  TCB_CHECK_ARG(out_mode != OUT_SPECTRUM || h->spectrum_ok,
                "tcb_fftfilter_apply: spectrum output needs n a power of two in [256, 4096]");
  TCB_CHECK_ARG(h->nkern == 1 || kern0 + nz <= h->nkern,
                "tcb_fftfilter_apply: kernel range [kern0, kern0+nz) exceeds nkern");
  Args a;
  a.x = x;
  a.ldx = ldx;
  a.xoff = xoff;
  a.nproj = (int)h->nproj;
  a.nz = (int)nz;
  a.half = (int)((nz + 1) / 2);
  a.n = (int)h->n;
  a.shared_kern = h->nkern == 1;
  a.kern0 = (int)kern0;
  a.H = h->H;
  a.AB = h->AB;
  a.twL = h->twL;
  a.twn = h->twn;
  a.out = out;
  a.ldo = ldo;
  const size_t blocks = (size_t)a.half * h->nproj;
  TCB_CHECK_ARG(blocks < (1ull << 31), "tcb_fftfilter_apply: too many rows");
  cudaStream_t s = (cudaStream_t)stream;
  StageTimer tm("fft_filter", s);
  switch (h->L) {
    case 256: launch<256>(a, out_mode, (unsigned)blocks, s); break;
    case 512: launch<512>(a, out_mode, (unsigned)blocks, s); break;
    case 1024: launch<1024>(a, out_mode, (unsigned)blocks, s); break;
    case 2048: launch<2048>(a, out_mode, (unsigned)blocks, s); break;
    case 4096: launch<4096>(a, out_mode, (unsigned)blocks, s); break;
    default: launch<8192>(a, out_mode, (unsigned)blocks, s); break;
  }
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

extern "C" int tcb_fftfilter_destroy(tcb_fftfilter *h) {
  if (!h) return TCB_OK;
  release(h);
  delete h;
  return TCB_OK;
}
