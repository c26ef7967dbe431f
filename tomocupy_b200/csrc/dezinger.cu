// Outlier (zinger) removal: ProcFunctions.remove_outliers
// (src/tomocupy/processing/proc_functions.py:96-107).  For frames
// [nframes, nz, n] (projections, darks or flats) and window width w:
//   f = median_filter(data, [w, 1, w])        (scipy/cupyx rank filter:
//        window rows i - w/2 .. i + (w-1)/2, mode 'reflect', rank (w*w)/2)
//   data = where(data > f and data - f > threshold, f, data)
// The window spans w frames and w columns of one detector row.  One thread
// per output pixel gathers its w*w values (as float: exact for 8/16-bit
// frames), sorts them with a bitonic network padded with +inf to a power of
// two, and takes the rank-(w*w)/2 value, so the result is the reference's
// bit for bit on integer frames.  Out of place (the window reads the
// original neighbours); the input may be a strided view (frame and row
// strides in elements), the output is contiguous [nframes, nz, n].
#include <cuda_fp16.h>

#include <cmath>

#include "common.cuh"

namespace tcb {
namespace {

// scipy 'reflect' (d c b a | a b c d | d c b a), periodic with period 2n
__device__ __forceinline__ int reflect_index(int i, int n) {
  if ((unsigned)i < (unsigned)n) return i;
  if (n == 1) return 0;
  const int p = 2 * n;
  i %= p;
  if (i < 0) i += p;
  return i < n ? i : p - 1 - i;
}

template <typename T>
__device__ __forceinline__ float load_val(const T *p) { return (float)__ldg(p); }

constexpr int pow2_at_least(int m) { return m <= 1 ? 1 : 2 * pow2_at_least((m + 1) / 2); }

// One thread per output pixel; W (the window width) is a template
// parameter so the W*W gather and the sorting network unroll completely
// and the window stays in registers.  The network is a bitonic sort of the
// W*W values padded with +inf to a power of two, with min/max
// compare-exchanges; the rank-(W*W)/2 entry is the median.
template <int W, typename T>
__global__ void __launch_bounds__(128) dezinger_kernel(T *__restrict__ out,
                                                       const T *__restrict__ in, int nframes,
                                                       int nz, int n, size_t fstride,
                                                       size_t zstride, float threshold) {
  constexpr int M = W * W, S = pow2_at_least(M);
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  const int f = blockIdx.z;
  if (x >= n) return;
  float v[S];
  int cx[W];
#pragma unroll
  for (int b = 0; b < W; b++) cx[b] = reflect_index(x - W / 2 + b, n);
#pragma unroll
  for (int a = 0; a < W; a++) {
    const T *r = in + (size_t)reflect_index(f - W / 2 + a, nframes) * fstride +
                 (size_t)z * zstride;
#pragma unroll
    for (int b = 0; b < W; b++) v[a * W + b] = load_val(r + cx[b]);
  }
#pragma unroll
  for (int q = M; q < S; q++) v[q] = INFINITY;
#pragma unroll
  for (int size = 2; size <= S; size <<= 1)
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
      for (int i = 0; i < S; i++) {
        const int j = i ^ stride;
        if (j > i) {
          const float lo = fminf(v[i], v[j]), hi = fmaxf(v[i], v[j]);
          if ((i & size) == 0) {
            v[i] = lo;
            v[j] = hi;
          } else {
            v[i] = hi;
            v[j] = lo;
          }
        }
      }
  const float med = v[M / 2];
  const T *ip = in + (size_t)f * fstride + (size_t)z * zstride + x;
  const T d = *ip;
  const float df = (float)d;
  out[((size_t)f * nz + z) * n + x] = (df > med && df - med > threshold) ? (T)med : d;
}

template <int W, typename T>
int launch(void *out, const void *in, int nframes, int nz, int n, size_t fs, size_t zs,
           float thr, cudaStream_t s) {
  dezinger_kernel<W, T><<<dim3(ceil_div(n, 128), nz, nframes), 128, 0, s>>>(
      (T *)out, (const T *)in, nframes, nz, n, fs, zs, thr);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

template <typename T>
int dispatch(void *out, const void *in, int nframes, int nz, int n, size_t fs, size_t zs, int w,
             float thr, cudaStream_t s) {
  switch (w) {
    case 1: return launch<1, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 2: return launch<2, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 3: return launch<3, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 4: return launch<4, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 5: return launch<5, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 6: return launch<6, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 7: return launch<7, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 8: return launch<8, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 9: return launch<9, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    case 10: return launch<10, T>(out, in, nframes, nz, n, fs, zs, thr, s);
    default: return launch<11, T>(out, in, nframes, nz, n, fs, zs, thr, s);
  }
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_dezinger(void *out, const void *in, int in_dtype, size_t nframes, size_t nz,
                            size_t n, size_t in_fstride, size_t in_zstride, int width,
                            double threshold, void *stream) {
  TCB_CHECK_ARG(out && in, "tcb_dezinger: null pointer");
  TCB_CHECK_ARG(out != in, "tcb_dezinger: out must not alias in");
  TCB_CHECK_ARG(width >= 1 && width <= 11, "tcb_dezinger: width %d not in [1, 11]", width);
  TCB_CHECK_ARG(nframes >= 1 && nframes <= 65535 && nz >= 1 && nz <= 65535 && n >= 1 &&
                    n < (1u << 30),
                "tcb_dezinger: bad sizes %zu x %zu x %zu", nframes, nz, n);
  TCB_CHECK_ARG(in_zstride >= n && in_fstride >= in_zstride * (nz - 1) + n,
                "tcb_dezinger: input strides make rows overlap");
  cudaStream_t s = (cudaStream_t)stream;
  StageTimer t("dezinger", s);
  // the reference compares data - f (in the frames' type) with the integer threshold
  const float thr = (float)threshold;
  switch (in_dtype) {
    case TCB_U8:
      return dispatch<uint8_t>(out, in, (int)nframes, (int)nz, (int)n, in_fstride, in_zstride,
                               width, thr, s);
    case TCB_U16:
      return dispatch<uint16_t>(out, in, (int)nframes, (int)nz, (int)n, in_fstride, in_zstride,
                                width, thr, s);
    case TCB_F32:
      return dispatch<float>(out, in, (int)nframes, (int)nz, (int)n, in_fstride, in_zstride,
                             width, thr, s);
    default: TCB_CHECK_ARG(false, "tcb_dezinger: unknown input type %d", in_dtype);
  }
}
