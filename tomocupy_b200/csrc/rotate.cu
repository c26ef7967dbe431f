// Projection rotation: ProcFunctions.rotate_proj
// (src/tomocupy/processing/proc_functions.py:126-138), which proc_proj applies
// after phase retrieval and before -log when rotate_proj_angle != 0
// (proc_functions.py:181-183): ndimage.rotate(data, angle, reshape=False,
// order=order, axes=(2, 1), mode='nearest') on [nproj, nz, n] stacks.
//
// ndimage.rotate is an affine map of every (z, x) plane: the output pixel
// (oz, ox) samples the input at
//   iz = (offz + oz * c) + ox * s,   ix = (offx + oz * (-s)) + ox * c
// (the rotation matrix [[c, s], [-s, c]] over the sorted axes (1, 2) and the
// offset that keeps the plane centre fixed), clamped to [0, len - 1]
// ('nearest'), then interpolated with B-spline weights of order 0 or 1
// (no prefilter below order 2).  The arithmetic is the published algorithm
// of scipy.ndimage's geometric transform, in float64 with every product and
// sum rounded separately (no fused multiply-add): the order-1 weights are
// (1 - t, 1 - (1 - t)), the terms v * wz * wx are accumulated in the order
// (z0, x0), (z0, x1), (z1, x0), (z1, x1) from 0, and the sum is rounded to
// float32 once.  The caller passes c, s and the offsets so that the host
// decides the trigonometry (the reference computes them with NumPy).
//
// One thread per output pixel (x fastest) and a run of frames: the float64
// coordinates and weights, the costly part, are formed once per pixel and
// reused for every frame of the run; for the small roll angles this
// corrects, a warp's four taps fall on two nearly contiguous row segments.
#include <algorithm>

#include "common.cuh"

namespace tcb {
namespace {

__device__ __forceinline__ double clamp_nearest(double c, int len) {
  // 'nearest' boundary: coordinates outside [0, len - 1] map to the edge
  if (c < 0.0) return 0.0;
  const double hi = (double)(len - 1);
  return c > hi ? hi : c;
}

template <int ORDER>
__global__ void __launch_bounds__(128) rotate_kernel(float *__restrict__ out,
                                                     const float *__restrict__ in, size_t nframes,
                                                     int nz, int n, size_t in_fstride,
                                                     size_t out_fstride, double c, double s,
                                                     double offz, double offx) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  if (x >= n) return;
  double iz = __dadd_rn(__dadd_rn(offz, __dmul_rn((double)z, c)), __dmul_rn((double)x, s));
  double ix = __dadd_rn(__dadd_rn(offx, __dmul_rn((double)z, -s)), __dmul_rn((double)x, c));
  iz = clamp_nearest(iz, nz);
  ix = clamp_nearest(ix, n);
  int z0, z1, x0, x1;
  double wz0 = 1.0, wz1 = 0.0, wx0 = 1.0, wx1 = 0.0;
  if (ORDER == 0) {
    z0 = min((int)floor(__dadd_rn(iz, 0.5)), nz - 1);
    x0 = min((int)floor(__dadd_rn(ix, 0.5)), n - 1);
    z1 = z0;
    x1 = x0;
  } else {
    const double fz = floor(iz), fx = floor(ix);
    z0 = (int)fz;
    x0 = (int)fx;
    wz0 = __dsub_rn(1.0, __dsub_rn(iz, fz));
    wz1 = __dsub_rn(1.0, wz0);
    wx0 = __dsub_rn(1.0, __dsub_rn(ix, fx));
    wx1 = __dsub_rn(1.0, wx0);
    z1 = min(z0 + 1, nz - 1);
    x1 = min(x0 + 1, n - 1);
  }
#pragma unroll 2
  for (size_t f = blockIdx.z; f < nframes; f += gridDim.z) {
    const float *p = in + f * in_fstride;
    double v;
    if (ORDER == 0) {
      v = (double)__ldg(p + (size_t)z0 * n + x0);
    } else {
      const float *r0 = p + (size_t)z0 * n, *r1 = p + (size_t)z1 * n;
      v = 0.0;
      v = __dadd_rn(v, __dmul_rn(__dmul_rn((double)__ldg(r0 + x0), wz0), wx0));
      v = __dadd_rn(v, __dmul_rn(__dmul_rn((double)__ldg(r0 + x1), wz0), wx1));
      v = __dadd_rn(v, __dmul_rn(__dmul_rn((double)__ldg(r1 + x0), wz1), wx0));
      v = __dadd_rn(v, __dmul_rn(__dmul_rn((double)__ldg(r1 + x1), wz1), wx1));
    }
    out[f * out_fstride + (size_t)z * n + x] = __double2float_rn(v);
  }
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_rotate_proj(float *out, const float *in, size_t nframes, size_t nz, size_t n,
                               size_t in_fstride, size_t out_fstride, double c, double s,
                               double offz, double offx, int order, void *stream) {
  TCB_CHECK_ARG(out && in && out != in, "tcb_rotate_proj: null or aliased pointers");
  TCB_CHECK_ARG(order == 0 || order == 1,
                "tcb_rotate_proj: spline order %d (orders 0 and 1 are supported)", order);
  TCB_CHECK_ARG(nframes >= 1 && nz >= 1 && nz <= 65535 && n >= 1 && n <= (1u << 30) &&
                    in_fstride >= nz * n && out_fstride >= nz * n,
                "tcb_rotate_proj: bad sizes nframes=%zu nz=%zu n=%zu strides=%zu/%zu", nframes,
                nz, n, in_fstride, out_fstride);
  cudaStream_t st = (cudaStream_t)stream;
  StageTimer t("rotate_proj", st);
  // frame runs: as few grid layers as keep about 64 CTAs per SM busy
  const size_t plane_ctas = (size_t)ceil_div(n, 128) * nz;
  const size_t layers = std::min<size_t>(
      {nframes, (size_t)65535, std::max<size_t>(1, ceil_div(148 * 64, plane_ctas))});
  const dim3 grid(ceil_div(n, 128), (unsigned)nz, (unsigned)layers);
  if (order == 0)
    rotate_kernel<0><<<grid, 128, 0, st>>>(out, in, nframes, (int)nz, (int)n, in_fstride,
                                           out_fstride, c, s, offz, offx);
  else
    rotate_kernel<1><<<grid, 128, 0, st>>>(out, in, nframes, (int)nz, (int)n, in_fstride,
                                           out_fstride, c, s, offz, offx);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}
