// Line (pixel-driven) backprojector for tomography and laminography.
//
// Same geometry and bilinear weights as cfunc_linerec
// (src/include/kernels_linerec.cuh:3-137): for voxel (tx, ty, tz) and angle t
//   u = cos(t)(x) + sin(t)(y) + n/2
//   v = sin(t)cos(phi)(x) - cos(t)cos(phi)(y) + sin(phi)(z) + nz/2
// with x = tx - n/2, y = ty - n/2, truncation (int)(u - 1e-5), and the
// output row flip f[tx + (n-1-ty) n + tz n^2] += 4/nproj * sum.
//
// B200 design: the per-angle rotation coefficients are computed once per CTA
// into shared memory (with the reference's __cosf/__sinf, so u and v are
// bit-identical) instead of by every thread for every angle; each thread
// accumulates in fp32 registers (also in the FLOAT16 variant, whose caller
// buffers are fp16); reads of the sinogram go through the read-only path.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <mutex>

#include "common.cuh"
#include "tcgen05.cuh"

struct tcb_linerec {
  size_t nproj, nz, n, ncproj, ncz;
  int precision;
  bool freed = false;
  int *err = nullptr;  // set by a TMA wait of backproject_full_tma that gave up
};

namespace tcb {
namespace lr {

constexpr int BX = 32, BY = 8;
constexpr int ACHUNK = 256;  // angles staged in shared memory per pass

enum Mode { FULL = 0, TRY = 1, TRY_LAMINO = 2 };

template <typename T> __device__ __forceinline__ float ld(const T *p) { return (float)*p; }
template <> __device__ __forceinline__ float ld<__half>(const __half *p) {
  return __half2float(*p);
}
template <typename T> __device__ __forceinline__ T from_f32(float v) { return (T)v; }
template <> __device__ __forceinline__ __half from_f32<__half>(float v) {
  return __float2half_rn(v);
}

// The reference kernel's arithmetic (kernels_linerec.cuh:23-40) with every
// rounding written out, so that no compiler contraction can differ from the
// reference build's: u = fma(R0, x, R1 y) + n/2,
// v = (fma(R3, x, R4 y) + R5 z) + nz/2 (R3 = sin(t) cos(phi),
// R4 = -cos(t) cos(phi); R5 z = sin(phi) z does not depend on the angle and
// is rounded on its own, as the reference's loop computes it), and the bilinear sum
// fma(d11, w11, fma(d10, w10, fma(d00, w00, d01 w01))) added to the
// accumulator.  Bit-identical per angle to the reference build.
__device__ __forceinline__ float lr_u(float R0, float R1, float x, float y, float h) {
  return __fadd_rn(__fmaf_rn(R0, x, __fmul_rn(R1, y)), h);
}
__device__ __forceinline__ float lr_v(float R3, float R4, float R5, float x, float y, float z,
                                      float hz) {
  return __fadd_rn(__fadd_rn(__fmaf_rn(R3, x, __fmul_rn(R4, y)), __fmul_rn(R5, z)), hz);
}
__device__ __forceinline__ float lr_interp(float d00, float d01, float d10, float d11, float u,
                                           float v) {
  const float w00 = __fmul_rn(1 - u, 1 - v), w01 = __fmul_rn(u, 1 - v);
  const float w10 = __fmul_rn(1 - u, v), w11 = __fmul_rn(u, v);
  return __fmaf_rn(d11, w11, __fmaf_rn(d10, w10, __fmaf_rn(d00, w00, __fmul_rn(d01, w01))));
}

template <typename T, int MODE>
__global__ void __launch_bounds__(BX *BY)
    backproject_kernel(T *__restrict__ f, const T *__restrict__ data,
                       const float *__restrict__ theta, float phi_s,
                       const float *__restrict__ phi_v, const float *__restrict__ sh,
                       float c, int sz, int ncz, int n, int nz, int nproj) {
  __shared__ float s_c[ACHUNK], s_s[ACHUNK];
  const int tx = blockIdx.x * BX + threadIdx.x;
  const int ty = blockIdx.y * BY + threadIdx.y;
  const int tz = blockIdx.z;
  const bool active = tx < n && ty < n && tz < ncz;
  const float phi = (MODE == TRY_LAMINO) ? (active ? phi_v[tz] : 0.f) : phi_s;
  const float cphi = __cosf(phi);
  const float sphi = __sinf(phi);
  const float shift = (MODE == TRY && active) ? sh[tz] : 0.f;
  const int zz = (MODE == FULL) ? (tz + sz - nz / 2) : (sz - nz / 2);
  float f0 = 0.f;
  const int tid = threadIdx.y * BX + threadIdx.x;
  for (int t0 = 0; t0 < nproj; t0 += ACHUNK) {
    int cnt = min(ACHUNK, nproj - t0);
    __syncthreads();
    for (int k = tid; k < cnt; k += BX * BY) {
      float th = theta[t0 + k];
      s_c[k] = __cosf(th);
      s_s[k] = __sinf(th);
    }
    __syncthreads();
    if (!active) continue;
    for (int k = 0; k < cnt; k++) {
      const int t = t0 + k;
      float ctheta = s_c[k];
      float stheta = s_s[k];
      float R0 = ctheta, R1 = stheta;
      float R3 = __fmul_rn(stheta, cphi), R4 = __fmul_rn(-ctheta, cphi), R5 = sphi;
      float u = lr_u(R0, R1, (float)(tx - n / 2), (float)(ty - n / 2), (float)(n / 2));
      if (MODE == TRY) u = __fsub_rn(u, shift);
      float v = lr_v(R3, R4, R5, (float)(tx - n / 2), (float)(ty - n / 2), (float)zz,
                     (float)(nz / 2));
      int ur = (int)(u - 1e-5f);
      int vr = (int)(v - 1e-5f);
      if ((ur >= 0) & (ur < n - 1) & (vr >= 0) & (vr < nz - 1)) {
        u = u - ur;
        v = v - vr;
        const T *d0 = data + ur + (size_t)t * n + (size_t)vr * n * nproj;
        const T *d1 = d0 + (size_t)n * nproj;
        f0 = __fadd_rn(f0, lr_interp(ld(d0), ld(d0 + 1), ld(d1), ld(d1 + 1), u, v));
      }
    }
  }
  if (!active) return;
  T *o = f + tx + (size_t)(n - ty - 1) * n + (size_t)tz * n * n;
  *o = from_f32<T>(__fmaf_rn(f0, c, ld(o)));
}

// FULL mode, ZS consecutive slices per thread, sinogram footprints staged in
// shared memory.  For each angle the CTA's 32 x 8 x ZS voxels read detector
// samples u in a window of at most 32|cos| + 8|sin| + 2 and, in tomography
// (cos(phi) ~ 0), rows vr in [tz0 + sz - 1, tz0 + sz + ZS]; a box of UW x VR
// samples per angle is loaded cooperatively for AC angles at a time.  Every
// voxel evaluates exactly the expressions of backproject_kernel (u, v, their
// truncation and weights) and reads the same sinogram values -- from the box
// when inside it, from global memory otherwise -- so the sums are
// bit-identical for any geometry; only the speed depends on the box holding
// the samples (tomography).
constexpr int ZS = 4;
constexpr int UW = 48, VR = ZS + 2, AC = 32;
template <typename T>
__global__ void __launch_bounds__(BX *BY)
    backproject_full_zs(T *__restrict__ f, const T *__restrict__ data,
                        const float *__restrict__ theta, float phi, float c, int sz, int ncz,
                        int n, int nz, int nproj) {
  __shared__ float s_c[AC], s_s[AC];
  __shared__ int s_u0[AC], s_v0[AC];
  __shared__ float box[AC][VR][UW];
  const int tx = blockIdx.x * BX + threadIdx.x;
  const int ty = blockIdx.y * BY + threadIdx.y;
  const int tz0 = blockIdx.z * ZS;
  const bool active = tx < n && ty < n;
  const float cphi = __cosf(phi);
  const float sphi = __sinf(phi);
  float acc[ZS];
#pragma unroll
  for (int s = 0; s < ZS; s++) acc[s] = 0.f;
  const int tid = threadIdx.y * BX + threadIdx.x;
  const int x0 = blockIdx.x * BX - n / 2, y0 = blockIdx.y * BY - n / 2;
  for (int t0 = 0; t0 < nproj; t0 += AC) {
    const int cnt = min(AC, nproj - t0);
    __syncthreads();
    if (tid < cnt) {
      float th = theta[t0 + tid];
      float ct = __cosf(th), st = __sinf(th);
      s_c[tid] = ct;
      s_s[tid] = st;
      // smallest u of the tile's corners, one sample of margin
      float umin = fminf(fminf(ct * x0 + st * y0, ct * (x0 + BX - 1) + st * y0),
                         fminf(ct * x0 + st * (y0 + BY - 1),
                               ct * (x0 + BX - 1) + st * (y0 + BY - 1))) + n / 2;
      s_u0[tid] = (int)floorf(umin) - 1;
      s_v0[tid] = tz0 + sz - 1;
    }
    __syncthreads();
    // stage the boxes: cnt x VR rows of UW samples (zeros outside the sinogram)
    for (int e = tid; e < cnt * VR * UW; e += BX * BY) {
      const int a = e / (VR * UW), r = (e / UW) % VR, w = e % UW;
      const int uu = s_u0[a] + w, vv = s_v0[a] + r;
      float val = 0.f;
      if (uu >= 0 && uu < n && vv >= 0 && vv < nz)
        val = ld(data + uu + (size_t)(t0 + a) * n + (size_t)vv * n * nproj);
      box[a][r][w] = val;
    }
    __syncthreads();
    if (!active) continue;
    for (int k = 0; k < cnt; k++) {
      const int t = t0 + k;
      float ctheta = s_c[k];
      float stheta = s_s[k];
      float R0 = ctheta, R1 = stheta;
      float R3 = __fmul_rn(stheta, cphi), R4 = __fmul_rn(-ctheta, cphi), R5 = sphi;
      float u = lr_u(R0, R1, (float)(tx - n / 2), (float)(ty - n / 2), (float)(n / 2));
      int ur = (int)(u - 1e-5f);
      if (!((ur >= 0) & (ur < n - 1))) continue;
      u = u - ur;
      const int bu = ur - s_u0[k];
      const bool uin = (bu >= 0) & (bu < UW - 1);
#pragma unroll
      for (int s = 0; s < ZS; s++) {
        const int tz = tz0 + s;
        const int zz = tz + sz - nz / 2;
        float v = lr_v(R3, R4, R5, (float)(tx - n / 2), (float)(ty - n / 2), (float)zz,
                     (float)(nz / 2));
        int vr = (int)(v - 1e-5f);
        if ((tz < ncz) & (vr >= 0) & (vr < nz - 1)) {
          v = v - vr;
          const int bv = vr - s_v0[k];
          float x00, x01, x10, x11;
          if (uin & (bv >= 0) & (bv < VR - 1)) {
            x00 = box[k][bv][bu];
            x01 = box[k][bv][bu + 1];
            x10 = box[k][bv + 1][bu];
            x11 = box[k][bv + 1][bu + 1];
          } else {
            const T *d0 = data + ur + (size_t)t * n + (size_t)vr * n * nproj;
            const T *d1 = d0 + (size_t)n * nproj;
            x00 = ld(d0);
            x01 = ld(d0 + 1);
            x10 = ld(d1);
            x11 = ld(d1 + 1);
          }
          acc[s] = __fadd_rn(acc[s], lr_interp(x00, x01, x10, x11, u, v));
        }
      }
    }
  }
  if (!active) return;
#pragma unroll
  for (int s = 0; s < ZS; s++) {
    const int tz = tz0 + s;
    if (tz >= ncz) break;
    T *o = f + tx + (size_t)(n - ty - 1) * n + (size_t)tz * n * n;
    *o = from_f32<T>(__fmaf_rn(acc[s], c, ld(o)));
  }
}

// FULL mode, float32, the same voxels, expressions and values as
// backproject_full_zs, with the per-angle sinogram boxes staged by TMA:
// a 3D tensor map over the sinogram (n, nproj, nz) and one box of TUW
// samples x 1 angle x VR rows per angle, its first sample rounded down to a
// multiple of 4 (16 bytes, the TMA alignment of the innermost coordinate;
// TUW = 48 + 4 keeps the window), zero-filled outside the sinogram.  Two
// stages of TAC angles: one thread issues the next chunk's TMA loads (one
// mbarrier per stage) while the CTA sums the current chunk, so the staging
// costs the CTA no load instructions and overlaps the arithmetic.  Every
// wait is bounded; a wait that gives up sets *err and the CTA stops.
constexpr int TUW = 52, TAC = 16;  // 16 angles per stage: 41 KB, 5 CTAs per SM
constexpr int TBOX = 1280;  // bytes per angle slot: TUW * VR * 4 = 1248, 128-byte aligned
constexpr int TSTAGE = TAC * TBOX;
constexpr int TSMEM = 2 * TSTAGE + 128;
static_assert(TUW * VR * 4 <= TBOX && TBOX % 128 == 0 && (TUW * 4) % 16 == 0, "TMA box");

__global__ void __launch_bounds__(BX *BY)
    backproject_full_tma(float *__restrict__ f, const float *__restrict__ data,
                         const __grid_constant__ CUtensorMap map,
                         const float *__restrict__ theta, float phi, float c, int sz, int ncz,
                         int n, int nz, int nproj, int *__restrict__ err) {
  using namespace tcb::tc;
  extern __shared__ uint8_t lr_raw[];
  uint8_t *sm = lr_raw + ((128u - (smem_u32(lr_raw) & 127u)) & 127u);
  __shared__ float s_c[2][TAC], s_s[2][TAC];
  __shared__ int s_u0[2][TAC];
  __shared__ uint64_t bar[2];
  const int tx = blockIdx.x * BX + threadIdx.x;
  const int ty = blockIdx.y * BY + threadIdx.y;
  const int tz0 = blockIdx.z * ZS;
  const bool active = tx < n && ty < n;
  const float cphi = __cosf(phi);
  const float sphi = __sinf(phi);
  float acc[ZS];
#pragma unroll
  for (int s = 0; s < ZS; s++) acc[s] = 0.f;
  const int tid = threadIdx.y * BX + threadIdx.x;
  const int x0 = blockIdx.x * BX - n / 2, y0 = blockIdx.y * BY - n / 2;
  const int v0 = tz0 + sz - 1;  // first sinogram row of every box
  const int nch = (nproj + TAC - 1) / TAC;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // rotation terms and box origins of chunk cc into stage st
  auto prep = [&](int cc, int st) {
    const int t0 = cc * TAC, cnt = min(TAC, nproj - t0);
    if (tid < cnt) {
      const float th = theta[t0 + tid];
      const float ct = __cosf(th), stt = __sinf(th);
      s_c[st][tid] = ct;
      s_s[st][tid] = stt;
      const float umin = fminf(fminf(ct * x0 + stt * y0, ct * (x0 + BX - 1) + stt * y0),
                               fminf(ct * x0 + stt * (y0 + BY - 1),
                                     ct * (x0 + BX - 1) + stt * (y0 + BY - 1))) +
                         n / 2;
      s_u0[st][tid] = ((int)floorf(umin) - 1) & ~3;  // down to a multiple of 4
    }
  };
  auto issue = [&](int cc, int st) {  // one thread
    const int t0 = cc * TAC, cnt = min(TAC, nproj - t0);
    mbar_expect_tx(&bar[st], (uint32_t)(cnt * TUW * VR * 4));
    for (int a = 0; a < cnt; a++)
      tma_load_3d(sm + st * TSTAGE + a * TBOX, &map, &bar[st], s_u0[st][a], t0 + a, v0);
  };
  prep(0, 0);
  __syncthreads();
  if (tid == 0) issue(0, 0);
  bool ok = true;
  int waited = 0;  // chunks whose stage barrier completed
  for (int cc = 0; cc < nch; cc++) {
    const int st = cc & 1;
    const int t0 = cc * TAC, cnt = min(TAC, nproj - t0);
    if (cc + 1 < nch) prep(cc + 1, st ^ 1);
    __syncthreads();
    if (tid == 0 && cc + 1 < nch) issue(cc + 1, st ^ 1);
    ok = __syncthreads_and(mbar_wait(&bar[st], (cc >> 1) & 1));
    if (!ok) break;
    waited = cc + 1;
    if (active) {
      for (int k = 0; k < cnt; k++) {
        const int t = t0 + k;
        float ctheta = s_c[st][k];
        float stheta = s_s[st][k];
        float R0 = ctheta, R1 = stheta;
        float R3 = __fmul_rn(stheta, cphi), R4 = __fmul_rn(-ctheta, cphi), R5 = sphi;
        float u = lr_u(R0, R1, (float)(tx - n / 2), (float)(ty - n / 2), (float)(n / 2));
        int ur = (int)(u - 1e-5f);
        if (!((ur >= 0) & (ur < n - 1))) continue;
        u = u - ur;
        const int bu = ur - s_u0[st][k];
        const bool uin = (bu >= 0) & (bu < TUW - 1);
        const float *bx = reinterpret_cast<const float *>(sm + st * TSTAGE + k * TBOX);
#pragma unroll
        for (int s = 0; s < ZS; s++) {
          const int tz = tz0 + s;
          const int zz = tz + sz - nz / 2;
          float v = lr_v(R3, R4, R5, (float)(tx - n / 2), (float)(ty - n / 2), (float)zz,
                     (float)(nz / 2));
          int vr = (int)(v - 1e-5f);
          if ((tz < ncz) & (vr >= 0) & (vr < nz - 1)) {
            v = v - vr;
            const int bv = vr - v0;
            float x00, x01, x10, x11;
            if (uin & (bv >= 0) & (bv < VR - 1)) {
              x00 = bx[bv * TUW + bu];
              x01 = bx[bv * TUW + bu + 1];
              x10 = bx[(bv + 1) * TUW + bu];
              x11 = bx[(bv + 1) * TUW + bu + 1];
            } else {
              const float *d0 = data + ur + (size_t)t * n + (size_t)vr * n * nproj;
              const float *d1 = d0 + (size_t)n * nproj;
              x00 = d0[0];
              x01 = d0[1];
              x10 = d1[0];
              x11 = d1[1];
            }
            acc[s] = __fadd_rn(acc[s], lr_interp(x00, x01, x10, x11, u, v));
          }
        }
      }
    }
    __syncthreads();  // stage st and its tables are refilled for chunk cc + 2
  }
  if (!ok) {
    // a wait gave up: report it, then wait (bounded) for the copies still in
    // flight (chunks waited .. waited + 1) before the CTA's smem goes away
    if (tid == 0) {
      atomicOr(err, 1);
      for (int cc = waited; cc < min(nch, waited + 2); cc++) mbar_wait(&bar[cc & 1], (cc >> 1) & 1);
    }
    __syncthreads();
    return;
  }
  if (!active) return;
#pragma unroll
  for (int s = 0; s < ZS; s++) {
    const int tz = tz0 + s;
    if (tz >= ncz) break;
    float *o = f + tx + (size_t)(n - ty - 1) * n + (size_t)tz * n * n;
    *o = __fmaf_rn(acc[s], c, *o);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 lr_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// The sinogram stack [nz][nproj][n] float32 as a TMA map with one
// TUW x 1 x VR box per angle; false when the layout does not allow it.
bool sino_map(CUtensorMap *m, const float *data, size_t n, size_t nproj, size_t nz) {
  auto fn = lr_encode_fn();
  if (!fn || n % 4 || ((uintptr_t)data & 15) || n < TUW) return false;
  cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)nproj, (cuuint64_t)nz};
  cuuint64_t strides[2] = {(cuuint64_t)(n * 4), (cuuint64_t)(n * nproj * 4)};
  cuuint32_t box[3] = {(cuuint32_t)TUW, 1, (cuuint32_t)VR};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(data), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T>
int launch(tcb_linerec *h, int mode, void *f, const void *g, const float *theta,
           float phi, const float *phi_v, const float *sh, int sz, cudaStream_t s) {
  dim3 blk(BX, BY), grd(ceil_div(h->n, BX), ceil_div(h->n, BY), (unsigned)h->ncz);
  StageTimer st("linerec", s);
  count_launch();
  float c = 4.0f / h->nproj;
  int n = (int)h->n, nz = (int)h->nz, ncz = (int)h->ncz, np = (int)h->ncproj;
  switch (mode) {
    case FULL: {
      dim3 grz(ceil_div(h->n, BX), ceil_div(h->n, BY), ceil_div(h->ncz, ZS));
      CUtensorMap map;
      // TCB_LINEREC_TMA=0 keeps the plain staging (for comparisons)
      const char *tsel = getenv("TCB_LINEREC_TMA");
      const bool tma_on = !(tsel && tsel[0] == '0');
      if (sizeof(T) == 4 && tma_on && h->err &&
          sino_map(&map, (const float *)g, h->n, h->ncproj, h->nz)) {
        backproject_full_tma<<<grz, blk, TSMEM, s>>>((float *)f, (const float *)g, map, theta,
                                                     phi, c, sz, ncz, n, nz, np, h->err);
        break;
      }
      backproject_full_zs<T><<<grz, blk, 0, s>>>((T *)f, (const T *)g, theta, phi, c, sz, ncz,
                                                  n, nz, np);
      break;
    }
    case TRY:
      backproject_kernel<T, TRY><<<grd, blk, 0, s>>>((T *)f, (const T *)g, theta, phi,
                                                     nullptr, sh, c, sz, ncz, n, nz, np);
      break;
    default:
      backproject_kernel<T, TRY_LAMINO><<<grd, blk, 0, s>>>(
          (T *)f, (const T *)g, theta, 0.f, phi_v, nullptr, c, sz, ncz, n, nz, np);
  }
  TCB_LAUNCH_CHECK();
  return TCB_OK;
}

int run(tcb_linerec *h, int mode, void *f, const void *g, const float *theta, float phi,
        const float *phi_v, const float *sh, int sz, void *stream) {
  TCB_CHECK_ARG(h, "linerec: null handle");
  TCB_CHECK_ARG(!h->freed, "linerec: handle was freed");
  TCB_CHECK_ARG(f && g && theta, "linerec: null pointer");
  TCB_CHECK_ARG(mode != TRY || sh, "linerec: backprojection_try needs sh");
  TCB_CHECK_ARG(mode != TRY_LAMINO || phi_v, "linerec: backprojection_try_lamino needs phi");
  if (h->precision == TCB_FLOAT16)
    return launch<__half>(h, mode, f, g, theta, phi, phi_v, sh, sz, (cudaStream_t)stream);
  return launch<float>(h, mode, f, g, theta, phi, phi_v, sh, sz, (cudaStream_t)stream);
}

}  // namespace lr
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_linerec_create(tcb_linerec **out, size_t nproj, size_t nz, size_t n,
                                  size_t ncproj, size_t ncz, int precision) {
  TCB_CHECK_ARG(out, "tcb_linerec_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 1 && nz >= 1 && n >= 2 && ncproj >= 1 && ncz >= 1,
                "tcb_linerec_create: bad sizes");
  TCB_CHECK_ARG(n < 65536 && ncz < 65536, "tcb_linerec_create: sizes too large");
  TCB_CHECK_ARG(precision == TCB_FLOAT32 || precision == TCB_FLOAT16,
                "tcb_linerec_create: bad precision %d", precision);
  tcb_linerec *h = new tcb_linerec();
  h->nproj = nproj;
  h->nz = nz;
  h->n = n;
  h->ncproj = ncproj;
  h->ncz = ncz;
  h->precision = precision;
  // the TMA-staged float32 kernel needs its dynamic shared memory and an
  // error flag; without them the plain kernel runs
  if (precision == TCB_FLOAT32 &&
      cudaFuncSetAttribute(lr::backproject_full_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           lr::TSMEM) == cudaSuccess &&
      cudaMalloc(&h->err, sizeof(int)) == cudaSuccess &&
      cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess) {
    cudaFree(h->err);
    h->err = nullptr;
  }
  cudaGetLastError();
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_linerec_status(tcb_linerec *h, int *timed_out) {
  TCB_CHECK_ARG(h && timed_out, "tcb_linerec_status: null pointer");
  *timed_out = 0;
  if (h->err) TCB_CUDA(cudaMemcpy(timed_out, h->err, sizeof(int), cudaMemcpyDeviceToHost));
  return TCB_OK;
}

extern "C" int tcb_linerec_backprojection(tcb_linerec *h, void *f, const void *g,
                                          const float *theta, float phi, int sz,
                                          void *stream) {
  return lr::run(h, lr::FULL, f, g, theta, phi, nullptr, nullptr, sz, stream);
}

extern "C" int tcb_linerec_backprojection_try(tcb_linerec *h, void *f, const void *g,
                                              const float *theta, const float *sh,
                                              float phi, int sz, void *stream) {
  return lr::run(h, lr::TRY, f, g, theta, phi, nullptr, sh, sz, stream);
}

extern "C" int tcb_linerec_backprojection_try_lamino(tcb_linerec *h, void *f,
                                                     const void *g, const float *theta,
                                                     const float *phi, int sz,
                                                     void *stream) {
  return lr::run(h, lr::TRY_LAMINO, f, g, theta, 0.f, phi, nullptr, sz, stream);
}

extern "C" int tcb_linerec_destroy(tcb_linerec *h) {
  if (!h) return TCB_OK;
  cudaFree(h->err);
  delete h;
  return TCB_OK;
}
