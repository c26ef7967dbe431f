// Binning of frames: utils.downsample (src/tomocupy/utils.py:157-167), which
// the reader applies to every chunk of projections, darks and flats after
// converting them to float32 (dataio/reader.py:335-356).  The reference
// halves the columns b times (x[::2] + x[1::2]) and then the rows b times,
// in float32; each output is the sum of a 2^b x 2^b block as a pairwise
// tree over its columns, then a pairwise tree over those row sums.  Here
// one thread per output pixel sums its block in exactly that order (the
// same float32 roundings, bit for bit; integer frames sum exactly).
#include "common.cuh"

namespace tcb {
namespace {

template <typename T>
__device__ __forceinline__ float ld(const T *p) { return (float)__ldg(p); }

template <int B, typename T>
__global__ void downsample_kernel(float *__restrict__ out, const T *__restrict__ in, int nz,
                                  int n, size_t fstride, size_t zstride) {
  constexpr int K = 1 << B;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  const int f = blockIdx.z;
  if (x >= n) return;
  float r[K];
#pragma unroll
  for (int i = 0; i < K; i++) {
    const T *row = in + (size_t)f * fstride + (size_t)(z * K + i) * zstride + (size_t)x * K;
    float c[K];
#pragma unroll
    for (int j = 0; j < K; j++) c[j] = ld(row + j);
#pragma unroll
    for (int w = K; w > 1; w >>= 1)
#pragma unroll
      for (int j = 0; j < w / 2; j++) c[j] = c[2 * j] + c[2 * j + 1];
    r[i] = c[0];
  }
#pragma unroll
  for (int w = K; w > 1; w >>= 1)
#pragma unroll
    for (int i = 0; i < w / 2; i++) r[i] = r[2 * i] + r[2 * i + 1];
  out[((size_t)f * nz + z) * n + x] = r[0];
}

template <int B, typename T>
int launch(float *out, const void *in, size_t nf, size_t nz, size_t n, size_t fs, size_t zs,
           cudaStream_t s) {
  downsample_kernel<B, T><<<dim3(ceil_div(n, 128), (unsigned)nz, (unsigned)nf), 128, 0, s>>>(
      out, (const T *)in, (int)nz, (int)n, fs, zs);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

template <typename T>
int dispatch(float *out, const void *in, size_t nf, size_t nz, size_t n, size_t fs, size_t zs,
             int b, cudaStream_t s) {
  switch (b) {
    case 1: return launch<1, T>(out, in, nf, nz, n, fs, zs, s);
    case 2: return launch<2, T>(out, in, nf, nz, n, fs, zs, s);
    case 3: return launch<3, T>(out, in, nf, nz, n, fs, zs, s);
    default: return launch<4, T>(out, in, nf, nz, n, fs, zs, s);
  }
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_downsample(float *out, const void *in, int in_dtype, size_t nframes, size_t nz,
                              size_t n, size_t in_fstride, size_t in_zstride, int binning,
                              void *stream) {
  TCB_CHECK_ARG(out && in, "tcb_downsample: null pointer");
  TCB_CHECK_ARG(binning >= 1 && binning <= 4, "tcb_downsample: binning %d not in [1, 4]",
                binning);
  TCB_CHECK_ARG(nframes >= 1 && nframes <= 65535 && nz >= 1 && nz <= 65535 && n >= 1,
                "tcb_downsample: bad sizes %zu x %zu x %zu", nframes, nz, n);
  const size_t K = (size_t)1 << binning;
  TCB_CHECK_ARG(in_zstride >= n * K && in_fstride >= in_zstride * (nz * K - 1) + n * K,
                "tcb_downsample: input strides too small for %zu x %zu binned output", nz, n);
  cudaStream_t s = (cudaStream_t)stream;
  StageTimer t("downsample", s);
  switch (in_dtype) {
    case TCB_U8: return dispatch<uint8_t>(out, in, nframes, nz, n, in_fstride, in_zstride, binning, s);
    case TCB_U16:
      return dispatch<uint16_t>(out, in, nframes, nz, n, in_fstride, in_zstride, binning, s);
    case TCB_F32: return dispatch<float>(out, in, nframes, nz, n, in_fstride, in_zstride, binning, s);
    default: TCB_CHECK_ARG(false, "tcb_downsample: unknown input type %d", in_dtype);
  }
}
