// Double-field-of-view padding: ProcFunctions.pad360
// (src/tomocupy/processing/proc_functions.py:109-124), applied after -log
// to every row of ni samples of a 360-degree scan whose rotation axis sits
// near one edge:
//   flip the row when the axis is on the left (centeri < ni // 2),
//   multiply its last w samples by the smooth transition v (float64, the
//   product rounded to float32), and zero-pad it to 2 * ni samples.
// Here in place on rows that already hold the ni samples at the start of a
// row of row_stride >= 2 * ni floats (the filter rows of the pipeline), one
// thread per output pair (x, ni - 1 - x) so the flip needs no scratch.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace tcb {
namespace {

__global__ void pad360_kernel(float *__restrict__ rows, const double *__restrict__ v, int ni,
                              size_t row_stride, int flip, int w) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // t in [0, ni): x = t (and its mirror)
  float *r = rows + (size_t)blockIdx.y * row_stride;
  const int half = (ni + 1) / 2;
  if (t < half) {
    const int a = t, b = ni - 1 - t;
    float va = r[a], vb = r[b];
    if (flip) {
      const float s = va;
      va = vb;
      vb = s;
    }
    // the transition covers columns [ni - w, ni)
    if (a >= ni - w) va = (float)((double)va * v[a - (ni - w)]);
    if (b != a && b >= ni - w) vb = (float)((double)vb * v[b - (ni - w)]);
    r[a] = va;
    r[b] = vb;
  }
  // zero padding [ni, 2 ni)
  if (t < ni) r[ni + t] = 0.f;
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_pad360_weights(double *v, size_t w) {
  TCB_CHECK_ARG(v && w >= 1, "tcb_pad360_weights: bad arguments");
  // v = linspace(1, 0, w, endpoint=False); v**5 * (126 - 420 v + 540 v**2 -
  // 315 v**3 + 70 v**4), with NumPy's float64 steps (v**2 a square, the
  // other integer powers through pow)
  const double step = (0.0 - 1.0) / (double)w;
  for (size_t j = 0; j < w; j++) {
    const double x = 1.0 + (double)j * step;
    const double p = 126.0 - 420.0 * x + 540.0 * (x * x) - 315.0 * std::pow(x, 3.0) +
                     70.0 * std::pow(x, 4.0);
    v[j] = std::pow(x, 5.0) * p;
  }
  return TCB_OK;
}

extern "C" int tcb_pad360_rows(float *rows, size_t nrows, size_t ni, size_t row_stride, int flip,
                               const double *v, size_t w, void *stream) {
  TCB_CHECK_ARG(rows && v, "tcb_pad360_rows: null pointer");
  TCB_CHECK_ARG(ni >= 1 && w >= 1 && w <= ni && row_stride >= 2 * ni && nrows >= 1 &&
                    nrows <= 65535u * 1024u,
                "tcb_pad360_rows: bad sizes nrows=%zu ni=%zu w=%zu stride=%zu", nrows, ni, w,
                row_stride);
  cudaStream_t s = (cudaStream_t)stream;
  StageTimer t("pad360", s);
  for (size_t r0 = 0; r0 < nrows; r0 += 65535) {
    const size_t nr = std::min<size_t>(65535, nrows - r0);
    pad360_kernel<<<dim3(ceil_div(ni, 256), (unsigned)nr), 256, 0, s>>>(
        rows + r0 * row_stride, v, (int)ni, row_stride, flip, (int)w);
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}
