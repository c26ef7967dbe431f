// Pre-processing kernels: dark/flat reductions and one fused pass that turns
// raw detector rows into (optionally -log'd, edge-padded) sinogram rows.
//
// Arithmetic follows ProcFunctions.darkflat_correction / minus_log
// (src/tomocupy/processing/proc_functions.py:55-83) operation by operation.
// Every CuPy elementwise step there is a separate kernel, so no multiply-add
// is ever contracted; the explicit __f*_rn intrinsics below keep nvcc from
// contracting either, which makes the fp32 results bit-identical.
#include <algorithm>
#include <cuda_fp16.h>

#include <mutex>

#include "common.cuh"

namespace tcb {
namespace {

template <typename T> __device__ __forceinline__ float to_f32(T v) { return (float)v; }

template <typename T>
__global__ void darkflat_stats_kernel(float *__restrict__ dark0, float *__restrict__ flat0,
                                      float *__restrict__ flat1,
                                      const T *__restrict__ dark, const T *__restrict__ flat,
                                      int ndark, int nflat, size_t plane, float bright_ratio,
                                      int flat_linear) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= plane) return;
  // dark0 = mean(dark, axis=0): float32 sum in frame order, then / count.
  float sd = 0.f;
  for (int k = 0; k < ndark; k++) sd = __fadd_rn(sd, to_f32(dark[(size_t)k * plane + i]));
  float d0 = __fdiv_rn(sd, (float)ndark);
  dark0[i] = d0;
  if (!flat_linear) {
    float sf = 0.f;
    for (int k = 0; k < nflat; k++)
      sf = __fadd_rn(sf, __fdiv_rn(to_f32(flat[(size_t)k * plane + i]), bright_ratio));
    float f0 = __fdiv_rn(sf, (float)nflat);
    f0 = __fmul_rn(f0, 1.00001f);  // cp.float32(1 + 1e-5)
    flat0[i] = __fsub_rn(f0, d0);
  } else {
    // flat0_p0 = mean(flat0[:nflat//2]), flat0_p1 = mean(flat0[nflat//2+1:])
    int h = nflat / 2;
    float s0 = 0.f, s1 = 0.f;
    for (int k = 0; k < h; k++)
      s0 = __fadd_rn(s0, __fdiv_rn(to_f32(flat[(size_t)k * plane + i]), bright_ratio));
    for (int k = h + 1; k < nflat; k++)
      s1 = __fadd_rn(s1, __fdiv_rn(to_f32(flat[(size_t)k * plane + i]), bright_ratio));
    flat0[i] = __fdiv_rn(s0, (float)h);
    flat1[i] = __fdiv_rn(s1, (float)(nflat - h - 1));
  }
}

struct PrepArgs {
  float *out;
  __half *hi, *lo;  // split-fp16 output planes (tcb_prep_rows_split16)
  const void *in;
  const float *dark0, *flat0, *flat1;
  int nproj, nz, n;
  size_t in_pstride, in_zstride;
  size_t out_zstride, out_pstride, out_poff, out_xoff, out_width;
  unsigned flags;
};

// -log with the reference's clean-up: where(x<=0 -> 1), log, negate,
// nan_to_num(nan=6, posinf=0, neginf=0).
__device__ __forceinline__ float minus_log(float x) {
  if (x <= 0.f) x = 1.f;
  float r = -logf(x);
  if (isnan(r)) r = 6.f;
  else if (isinf(r)) r = 0.f;
  return r;
}

// Apply the normalisation chain to one raw value.  d0/f0/f1 are the
// dark/flat statistics of this (z, x) position.
__device__ __forceinline__ float prep_apply(unsigned flags, float v, float d0, float f0,
                                            float f1, double vlin) {
  if (flags & TCB_PREP_DARKFLAT) {
    if (flags & TCB_PREP_FLAT_LINEAR) {
      // float64 path of the reference: (1-v)*p0 + v*p1, *= f32(1+1e-5), -= dark0
      double f = __dadd_rn(__dmul_rn(__dsub_rn(1.0, vlin), (double)f0),
                           __dmul_rn(vlin, (double)f1));
      f = __dmul_rn(f, (double)1.00001f);
      f = __dsub_rn(f, (double)d0);
      v = (float)__ddiv_rn((double)__fsub_rn(v, d0), f);
    } else {
      v = __fdiv_rn(__fsub_rn(v, d0), f0);
    }
  }
  if (flags & TCB_PREP_MINUS_LOG) v = minus_log(v);
  return v;
}

template <typename T> struct Vec4Of;
template <> struct Vec4Of<uint16_t> { using type = ushort4; };
template <> struct Vec4Of<uint8_t> { using type = uchar4; };
template <> struct Vec4Of<float> { using type = float4; };

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

template <typename T>
__device__ __forceinline__ float prep_scalar(const PrepArgs &a, const T *src, int z, int x,
                                             double vlin) {
  size_t i = (size_t)z * a.n + x;
  float d0 = 0.f, f0 = 1.f, f1 = 0.f;
  if (a.flags & TCB_PREP_DARKFLAT) {
    d0 = a.dark0[i];
    f0 = a.flat0[i];
    if (a.flags & TCB_PREP_FLAT_LINEAR) f1 = a.flat1[i];
  }
  return prep_apply(a.flags, to_f32(src[x]), d0, f0, f1, vlin);
}

// v = hi + lo with hi = fp16(v) and lo = fp16(v - hi): 22 significant bits
// in two fp16 planes, the operand format of the tensor-core filter.
__device__ __forceinline__ void split16(float v, __half &h, __half &l) {
  h = __float2half_rn(v);
  l = __float2half_rn(__fsub_rn(v, __half2float(h)));
}

// Output rows (z, p) enumerated z-major, a CTA taking rows blockIdx.x,
// blockIdx.x + gridDim.x, ... (a row is 2 n bytes in and 4 n out: too short
// for a CTA of its own).  SPLIT writes the row as two fp16 planes (hi, lo)
// instead of fp32.
template <typename T, bool SPLIT>
__device__ __forceinline__ void prep_one_row(const PrepArgs &a, size_t row);

template <typename T, bool SPLIT>
__global__ void __launch_bounds__(256) prep_rows_kernel(PrepArgs a) {
  const size_t rows = (size_t)a.nproj * a.nz;
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x) prep_one_row<T, SPLIT>(a, row);
}

template <typename T, bool SPLIT>
__device__ __forceinline__ void prep_one_row(const PrepArgs &a, size_t row) {
  int z = (int)(row / a.nproj);
  int p = (int)(row % a.nproj);
  const T *src = (const T *)a.in + (size_t)p * a.in_pstride + (size_t)z * a.in_zstride;
  const size_t orow = (size_t)z * a.out_zstride + (size_t)(p + a.out_poff) * a.out_pstride;
  float *dst = SPLIT ? nullptr : a.out + orow;
  __half *dhi = SPLIT ? a.hi + orow + a.out_xoff : nullptr;
  __half *dlo = SPLIT ? a.lo + orow + a.out_xoff : nullptr;
  double vlin = 0.0;
  if (a.flags & TCB_PREP_FLAT_LINEAR)
    vlin = (p == a.nproj - 1) ? 1.0 : __dmul_rn((double)p, 1.0 / (double)(a.nproj - 1));
  const int n = a.n;
  float *row_out = SPLIT ? nullptr : dst + a.out_xoff;
  const bool df = (a.flags & TCB_PREP_DARKFLAT) != 0;
  const bool lin = (a.flags & TCB_PREP_FLAT_LINEAR) != 0;
  const bool out_al = SPLIT ? ((((uintptr_t)dhi) & 7) == 0 && (((uintptr_t)dlo) & 7) == 0)
                            : ((((uintptr_t)row_out) & 15) == 0);
  // Vector path: 4 elements per thread per step when everything is aligned.
  bool vec = (n % 4 == 0) && out_al &&
             ((((uintptr_t)src) & (sizeof(T) * 4 - 1)) == 0) &&
             (!df || ((((uintptr_t)(a.dark0 + (size_t)z * n)) & 15) == 0 &&
                      (((uintptr_t)(a.flat0 + (size_t)z * n)) & 15) == 0 &&
                      (!lin || (((uintptr_t)(a.flat1 + (size_t)z * n)) & 15) == 0)));
  if (vec) {
    using V = typename Vec4Of<T>::type;
    for (int x = threadIdx.x * 4; x < n; x += blockDim.x * 4) {
      V raw = *reinterpret_cast<const V *>(src + x);
      float4 d0 = make_float4(0.f, 0.f, 0.f, 0.f), f0 = make_float4(1.f, 1.f, 1.f, 1.f),
             f1 = d0;
      if (df) {
        size_t i = (size_t)z * n + x;
        d0 = ld4(a.dark0 + i);
        f0 = ld4(a.flat0 + i);
        if (lin) f1 = ld4(a.flat1 + i);
      }
      float4 r;
      r.x = prep_apply(a.flags, (float)raw.x, d0.x, f0.x, f1.x, vlin);
      r.y = prep_apply(a.flags, (float)raw.y, d0.y, f0.y, f1.y, vlin);
      r.z = prep_apply(a.flags, (float)raw.z, d0.z, f0.z, f1.z, vlin);
      r.w = prep_apply(a.flags, (float)raw.w, d0.w, f0.w, f1.w, vlin);
      if constexpr (SPLIT) {
        __half h[4], l[4];
        split16(r.x, h[0], l[0]);
        split16(r.y, h[1], l[1]);
        split16(r.z, h[2], l[2]);
        split16(r.w, h[3], l[3]);
        *reinterpret_cast<uint2 *>(dhi + x) = *reinterpret_cast<const uint2 *>(h);
        *reinterpret_cast<uint2 *>(dlo + x) = *reinterpret_cast<const uint2 *>(l);
      } else {
        *reinterpret_cast<float4 *>(row_out + x) = r;
      }
    }
  } else {
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
      float v = prep_scalar<T>(a, src, z, x, vlin);
      if constexpr (SPLIT) split16(v, dhi[x], dlo[x]);
      else row_out[x] = v;
    }
  }
  if (!SPLIT && (a.flags & TCB_PREP_EDGE_PAD)) {
    float left = prep_scalar<T>(a, src, z, 0, vlin);
    float right = prep_scalar<T>(a, src, z, n - 1, vlin);
    size_t xo = a.out_xoff, xe = a.out_xoff + n;
    for (size_t x = threadIdx.x; x < xo; x += blockDim.x) dst[x] = left;
    for (size_t x = xe + threadIdx.x; x < a.out_width; x += blockDim.x) dst[x] = right;
  }
}

// CTAs for `rows` output rows: 16 per SM of 148 (each loops over rows)
inline unsigned prep_grid(size_t rows) { return (unsigned)std::min<size_t>(rows, 148 * 16); }

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_darkflat_stats(void *dark0, void *flat0, void *flat1, const void *dark,
                                  const void *flat, size_t ndark, size_t nflat, size_t nz,
                                  size_t n, int in_dtype, float bright_ratio,
                                  int flat_linear, void *stream) {
  TCB_CHECK_ARG(dark0 && flat0 && dark && flat, "tcb_darkflat_stats: null pointer");
  TCB_CHECK_ARG(ndark >= 1 && nflat >= 1, "tcb_darkflat_stats: need >=1 dark and flat");
  TCB_CHECK_ARG(!flat_linear || (nflat >= 3 && flat1),
                "tcb_darkflat_stats: flat_linear needs >=3 flats and flat1");
  size_t plane = nz * n;
  if (plane == 0) return TCB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned grid = ceil_div(plane, 256);
  StageTimer st("darkflat_stats", s);
  count_launch();
  switch (in_dtype) {
    case TCB_U16:
      darkflat_stats_kernel<uint16_t><<<grid, 256, 0, s>>>(
          (float *)dark0, (float *)flat0, (float *)flat1, (const uint16_t *)dark,
          (const uint16_t *)flat, (int)ndark, (int)nflat, plane, bright_ratio, flat_linear);
      break;
    case TCB_U8:
      darkflat_stats_kernel<uint8_t><<<grid, 256, 0, s>>>(
          (float *)dark0, (float *)flat0, (float *)flat1, (const uint8_t *)dark,
          (const uint8_t *)flat, (int)ndark, (int)nflat, plane, bright_ratio, flat_linear);
      break;
    case TCB_F32:
      darkflat_stats_kernel<float><<<grid, 256, 0, s>>>(
          (float *)dark0, (float *)flat0, (float *)flat1, (const float *)dark,
          (const float *)flat, (int)ndark, (int)nflat, plane, bright_ratio, flat_linear);
      break;
    default:
      set_error("tcb_darkflat_stats: unknown dtype %d", in_dtype);
      return TCB_ERR_INVALID_ARGUMENT;
  }
  TCB_LAUNCH_CHECK();
  return TCB_OK;
}

extern "C" int tcb_prep_rows(float *out, const void *in, const float *dark0,
                             const float *flat0, const float *flat1, size_t nproj,
                             size_t nz, size_t n, size_t in_pstride, size_t in_zstride,
                             int in_dtype, size_t out_zstride, size_t out_pstride,
                             size_t out_poff, size_t out_xoff, size_t out_width,
                             unsigned flags, void *stream) {
  TCB_CHECK_ARG(out && in, "tcb_prep_rows: null pointer");
  TCB_CHECK_ARG(!(flags & TCB_PREP_DARKFLAT) || (dark0 && flat0),
                "tcb_prep_rows: darkflat needs dark0/flat0");
  TCB_CHECK_ARG(!(flags & TCB_PREP_FLAT_LINEAR) || (flat1 && nproj >= 2),
                "tcb_prep_rows: flat_linear needs flat1 and nproj>=2");
  TCB_CHECK_ARG(out_width >= out_xoff + n || !(flags & TCB_PREP_EDGE_PAD),
                "tcb_prep_rows: out_width < out_xoff + n");
  TCB_CHECK_ARG(nproj < (1u << 31) && nz < (1u << 31) && n < (1u << 31),
                "tcb_prep_rows: size too large");
  if (nproj == 0 || nz == 0 || n == 0) return TCB_OK;
  size_t rows = nproj * nz;
  TCB_CHECK_ARG(rows < (1ull << 31), "tcb_prep_rows: too many rows in one call");
  PrepArgs a{out, nullptr, nullptr, in, dark0, flat0, flat1, (int)nproj, (int)nz, (int)n,
             in_pstride, in_zstride, out_zstride, out_pstride, out_poff, out_xoff, out_width,
             flags};
  cudaStream_t s = (cudaStream_t)stream;
  StageTimer st("prep_rows", s);
  count_launch();
  switch (in_dtype) {
    case TCB_U16: prep_rows_kernel<uint16_t, false><<<prep_grid(rows), 256, 0, s>>>(a); break;
    case TCB_U8: prep_rows_kernel<uint8_t, false><<<prep_grid(rows), 256, 0, s>>>(a); break;
    case TCB_F32: prep_rows_kernel<float, false><<<prep_grid(rows), 256, 0, s>>>(a); break;
    default:
      set_error("tcb_prep_rows: unknown dtype %d", in_dtype);
      return TCB_ERR_INVALID_ARGUMENT;
  }
  TCB_LAUNCH_CHECK();
  return TCB_OK;
}

extern "C" int tcb_prep_rows_split16(void *hi, void *lo, const void *in, const float *dark0,
                                     const float *flat0, const float *flat1, size_t nproj,
                                     size_t nz, size_t n, size_t in_pstride,
                                     size_t in_zstride, int in_dtype, size_t out_zstride,
                                     size_t out_pstride, unsigned flags, void *stream) {
  TCB_CHECK_ARG(hi && lo && in, "tcb_prep_rows_split16: null pointer");
  TCB_CHECK_ARG(!(flags & TCB_PREP_DARKFLAT) || (dark0 && flat0),
                "tcb_prep_rows_split16: darkflat needs dark0/flat0");
  TCB_CHECK_ARG(!(flags & TCB_PREP_FLAT_LINEAR) || (flat1 && nproj >= 2),
                "tcb_prep_rows_split16: flat_linear needs flat1 and nproj>=2");
  TCB_CHECK_ARG(!(flags & TCB_PREP_EDGE_PAD),
                "tcb_prep_rows_split16: edge padding is folded into the filter operator");
  TCB_CHECK_ARG(out_pstride >= n, "tcb_prep_rows_split16: out_pstride < n");
  TCB_CHECK_ARG(nproj < (1u << 31) && nz < (1u << 31) && n < (1u << 31),
                "tcb_prep_rows_split16: size too large");
  if (nproj == 0 || nz == 0 || n == 0) return TCB_OK;
  size_t rows = nproj * nz;
  TCB_CHECK_ARG(rows < (1ull << 31), "tcb_prep_rows_split16: too many rows in one call");
  PrepArgs a{nullptr, (__half *)hi, (__half *)lo, in, dark0, flat0, flat1, (int)nproj,
             (int)nz, (int)n, in_pstride, in_zstride, out_zstride, out_pstride, 0, 0, n,
             flags};
  cudaStream_t s = (cudaStream_t)stream;
  StageTimer st("prep_rows", s);
  count_launch();
  switch (in_dtype) {
    case TCB_U16: prep_rows_kernel<uint16_t, true><<<prep_grid(rows), 256, 0, s>>>(a); break;
    case TCB_U8: prep_rows_kernel<uint8_t, true><<<prep_grid(rows), 256, 0, s>>>(a); break;
    case TCB_F32: prep_rows_kernel<float, true><<<prep_grid(rows), 256, 0, s>>>(a); break;
    default:
      set_error("tcb_prep_rows_split16: unknown dtype %d", in_dtype);
      return TCB_ERR_INVALID_ARGUMENT;
  }
  TCB_LAUNCH_CHECK();
  return TCB_OK;
}

// ---------------------------------------------------------------------------
// Frame normalisation without any device allocation.
//
// Some callers cannot allocate device memory at the point where they
// normalise frames: acquisition loops that must not allocate once streaming
// has started, code running inside another runtime that owns the device
// allocator, or work recorded into a CUDA graph.  tcb_prep_rows needs the
// dark/flat statistics in caller-provided device buffers; this entry point
// keeps them in a fixed array in the library's own device memory instead.
// The array holds 2 * TCB_NOALLOC_MAX_PLANE floats (8 MiB) on every device
// that loads the library, for the life of the process.  All calls share it,
// so calls that overlap on the GPU (different streams or threads) race; each
// call rewrites every statistic it uses, so nothing is carried over from the
// previous call.  The first call on a device looks up the array's device
// address (cudaGetSymbolAddress) with that device current; make that first
// call before any stream capture.
namespace tcb {
namespace {
__device__ __align__(256) float g_noalloc_stats[2 * TCB_NOALLOC_MAX_PLANE];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float *g_noalloc_ptr[kMaxDevices] = {};

int noalloc_stats_ptr(float **out) {
  int dev = 0;
  TCB_CUDA(cudaGetDevice(&dev));
  TCB_CHECK_ARG(dev >= 0 && dev < kMaxDevices, "tcb_prep_noalloc: device index %d", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    TCB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_stats));
    g_noalloc_ptr[dev] = static_cast<float *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return TCB_OK;
}
}  // namespace
}  // namespace tcb

extern "C" int tcb_prep_noalloc(float *out, const void *data, const void *dark,
                                const void *flat, size_t nproj, size_t nz, size_t n,
                                size_t ndark, size_t nflat, int in_dtype, float bright_ratio,
                                size_t out_zstride, size_t out_pstride, size_t out_poff,
                                size_t out_xoff, size_t out_width, unsigned flags,
                                void *stream) {
  TCB_CHECK_ARG(out && data && dark && flat, "tcb_prep_noalloc: null pointer");
  TCB_CHECK_ARG(ndark >= 1 && nflat >= 1, "tcb_prep_noalloc: need >=1 dark and flat");
  TCB_CHECK_ARG(!(flags & TCB_PREP_FLAT_LINEAR),
                "tcb_prep_noalloc: flat_linear is not supported without allocation");
  TCB_CHECK_ARG((flags & ~(unsigned)(TCB_PREP_DARKFLAT | TCB_PREP_MINUS_LOG |
                                     TCB_PREP_EDGE_PAD)) == 0,
                "tcb_prep_noalloc: unknown flags 0x%x", flags);
  TCB_CHECK_ARG(nz * n <= (size_t)TCB_NOALLOC_MAX_PLANE,
                "tcb_prep_noalloc: nz*n = %zu exceeds the fixed scratch of %u elements; "
                "split the rows into smaller chunks or use tcb_prep_rows",
                nz * n, (unsigned)TCB_NOALLOC_MAX_PLANE);
  TCB_CHECK_ARG(!(flags & TCB_PREP_EDGE_PAD) || out_width >= out_xoff + n,
                "tcb_prep_noalloc: out_width < out_xoff + n");
  TCB_CHECK_ARG(nproj < (1u << 31) && nproj * nz < (1ull << 31),
                "tcb_prep_noalloc: too many rows in one call");
  TCB_CHECK_ARG(in_dtype == TCB_U16 || in_dtype == TCB_U8 || in_dtype == TCB_F32,
                "tcb_prep_noalloc: unknown dtype %d", in_dtype);
  if (nproj == 0 || nz == 0 || n == 0) return TCB_OK;
  float *stats = nullptr;
  int st = noalloc_stats_ptr(&stats);
  if (st != TCB_OK) return st;
  float *dark0 = stats, *flat0 = stats + TCB_NOALLOC_MAX_PLANE;
  size_t plane = nz * n;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned sgrid = ceil_div(plane, 256);
  PrepArgs a{out, nullptr, nullptr, data, dark0, flat0, nullptr, (int)nproj, (int)nz, (int)n,
             nz * n, n, out_zstride, out_pstride, out_poff, out_xoff, out_width,
             flags | TCB_PREP_DARKFLAT};
  const size_t rows = nproj * nz;
  StageTimer t("prep_noalloc", s);
  switch (in_dtype) {
    case TCB_U16:
      darkflat_stats_kernel<uint16_t><<<sgrid, 256, 0, s>>>(
          dark0, flat0, nullptr, (const uint16_t *)dark, (const uint16_t *)flat, (int)ndark,
          (int)nflat, plane, bright_ratio, 0);
      TCB_LAUNCH_CHECK();
      prep_rows_kernel<uint16_t, false><<<prep_grid(rows), 256, 0, s>>>(a);
      break;
    case TCB_U8:
      darkflat_stats_kernel<uint8_t><<<sgrid, 256, 0, s>>>(
          dark0, flat0, nullptr, (const uint8_t *)dark, (const uint8_t *)flat, (int)ndark,
          (int)nflat, plane, bright_ratio, 0);
      TCB_LAUNCH_CHECK();
      prep_rows_kernel<uint8_t, false><<<prep_grid(rows), 256, 0, s>>>(a);
      break;
    default:
      darkflat_stats_kernel<float><<<sgrid, 256, 0, s>>>(
          dark0, flat0, nullptr, (const float *)dark, (const float *)flat, (int)ndark,
          (int)nflat, plane, bright_ratio, 0);
      TCB_LAUNCH_CHECK();
      prep_rows_kernel<float, false><<<prep_grid(rows), 256, 0, s>>>(a);
  }
  TCB_LAUNCH_CHECK();
  count_launch(2);
  return TCB_OK;
}
