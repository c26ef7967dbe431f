// Tensor-core filter: the reference's ramp/window filter with the centre
// phase ramp, edge padding and crop (BackprojFunctions.fbp_filter_center,
// src/tomocupy/reconstruction/backproj_functions.py:93-109, and
// cfunc_filter::filter, src/cuda/cfunc_filter.cu:49-61) applied as one
// fp16 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulators in TMEM,
// operands staged by TMA).
//
// Why a GEMM.  The reference edge-pads each row of n samples to ne = 4n,
// multiplies its spectrum by w (filter x phase ramp), and crops n samples.
// That chain is linear in the n input samples, so it is an n x n matrix per
// filter kernel:
//   y[j] = sum_m hz[(pad + j - m) mod ne] * xpad[m],   hz = C2R(w) (unnormalised)
// which is Toeplitz, T[j][i] = hz[(j - i) mod ne], except that the edge
// padding folds the left pad into column 0 and the right pad into column n-1:
//   T[j][0]   = sum_{d=j}^{j+pad} hz[d]
//   T[j][n-1] = sum_{d=j+pad-ne+1}^{j-n+1} hz[d mod ne].
// A row of the sinogram then costs 2 n^2 tensor-core flops instead of two
// padded 4n-point FFTs and a spectral multiply that stream 4x the data.
//
// Precision.  Operands are fp16 with a split-precision correction:
// x = x_hi + x_lo and T*2^s = T_hi + T_lo (each fp16), and
//   y*2^s = x_hi T_hi + x_lo T_hi + x_hi T_lo
// accumulated in fp32 in TMEM (the dropped x_lo T_lo term is 2^-22 relative).
// The three products are one K loop of 3*n over [A_hi|A_lo|A_hi] x
// [B_hi|B_hi|B_lo].  2^s scales T into fp16's normal range; the epilogue
// multiplies by 2^-s.  T is built in float64 from float64 hz.
//
// Kernel shape: one 128 x 256 output tile per CTA (128 sinogram rows of one
// slice x 256 detector columns), K blocks of 64 in a 4-stage TMA ring
// (48 KB per stage, SWIZZLE_128B), one thread issuing TMA, one issuing MMA,
// all four warps draining TMEM in the epilogue.  Every mbarrier wait is
// bounded by a clock budget; a wait that runs out sets the handle's error
// flag and the CTA finishes without further waits.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "tcgen05.cuh"

struct tcb_tcfilter {
  size_t nproj, nz, n, nkern;
  int npad, kpad;         // B rows per kernel (multiple of 256), K extent (multiple of 64)
  __half *thi, *tlo;      // [nkern * npad][kpad]
  float inv_scale;
  int *err;               // device flag set by a timed-out wait
  bool ready;
};

namespace tcb {
namespace tcf {
using namespace tcb::tc;

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;
constexpr int B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t TMEM_COLS = 256;
constexpr uint32_t IDESC = tc::idesc_f16_f32(BM, BN);  // M = 128, N = 256

enum { OUT_ROWS = 0, OUT_PAIRS = 1 };

struct GemmArgs {
  float *out;
  size_t ldo;
  int nproj, nz, n, zh;
  int ptiles, ntn, kblocks, npad;
  int shared_kern, kern0;
  float inv_scale;
  int *err;
};

template <int MODE>
__global__ void __launch_bounds__(128, 1)
    tcf_gemm(const __grid_constant__ CUtensorMap ma_hi, const __grid_constant__ CUtensorMap ma_lo,
             const __grid_constant__ CUtensorMap mb_hi, const __grid_constant__ CUtensorMap mb_lo,
             const GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t base_u32 = smem_u32(smem_raw);
  uint8_t *smem = smem_raw + ((1024u - (base_u32 & 1023u)) & 1023u);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nt = blockIdx.x % g.ntn;
  const int mt = blockIdx.x / g.ntn;
  int z, ptile;
  if (MODE == OUT_PAIRS) {  // slices z and z + nz/2 of one angle tile run back to back
    const int c = mt & 1, r = mt >> 1;
    ptile = r % g.ptiles;
    z = r / g.ptiles + c * g.zh;
  } else {
    ptile = mt % g.ptiles;
    z = mt / g.ptiles;
  }
  const int p0 = ptile * BM;
  const int arow = z * g.nproj + p0;
  const int kern = g.shared_kern ? 0 : g.kern0 + z;
  const int brow = kern * g.npad + nt * BN;

  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int total = 3 * g.kblocks;
  bool ok = true;
  if (tid == 0) {
    // TMA producer: segment 0 = (A_hi, B_hi), 1 = (A_lo, B_hi), 2 = (A_hi, B_lo)
    for (int kb = 0; kb < total; kb++) {
      const int s = kb % STAGES, round = kb / STAGES;
      if (kb >= STAGES && !mbar_wait(&empty[s], (round - 1) & 1)) {
        ok = false;
        break;
      }
      const int seg = kb / g.kblocks;
      const int k0 = (kb % g.kblocks) * BK;
      uint8_t *sa = smem + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      tma_load_2d(sa, seg == 1 ? &ma_lo : &ma_hi, &full[s], k0, arow);
      tma_load_2d(sa + A_BYTES, seg == 2 ? &mb_lo : &mb_hi, &full[s], k0, brow);
    }
  } else if (tid == 32) {
    // MMA issuer: 4 x (128 x 256 x 16) per K block, then release the stage.
    for (int kb = 0; kb < total; kb++) {
      const int s = kb % STAGES, round = kb / STAGES;
      if (!mbar_wait(&full[s], round & 1)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(smem + s * STAGE_BYTES), sb = sa + A_BYTES;
#pragma unroll
      for (int k = 0; k < BK / 16; k++)
        mma_f16(tmem, sdesc(sa + k * 32), sdesc(sb + k * 32), IDESC, (kb > 0 || k > 0) ? 1u : 0u);
      mma_commit(&empty[s]);
    }
    mma_commit(done);
  }
  __syncwarp();
  if (!mbar_wait(done, 0)) ok = false;
  __syncwarp();
  tc_fence_after();

  // Epilogue: warp w owns accumulator rows (TMEM lanes) 32w .. 32w+31.  Each
  // 32 x 32 block goes through shared memory (the pipeline buffers are idle
  // now) so that one warp store covers 32 consecutive columns of one row.
  float *tb = reinterpret_cast<float *>(smem) + warp * (32 * 33);
  const bool wok = __all_sync(0xffffffffu, ok) && z < g.nz;
  for (int c0 = 0; c0 < BN; c0 += 32) {
    float v[32];
    tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
    for (int i = 0; i < 32; i++) tb[i * 33 + lane] = v[i];
    __syncwarp();
    const int j = nt * BN + c0 + lane;
    if (wok && nt * BN + c0 < g.n) {
      const int q = z % g.zh, comp = z / g.zh;
#pragma unroll 4
      for (int r = 0; r < 32; r++) {
        const int p = p0 + warp * 32 + r;
        if (p >= g.nproj || j >= g.n) continue;
        const float val = tb[lane * 33 + r] * g.inv_scale;
        if (MODE == OUT_ROWS)
          g.out[((size_t)z * g.nproj + p) * g.ldo + j] = val;
        else
          g.out[(((size_t)q * g.nproj + p) * g.n + j) * 2 + comp] = val;
      }
    }
    __syncwarp();
  }
  if (!ok) atomicOr(g.err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

// T_hi / T_lo of every kernel from float64 hz and the two folded edge columns.
__global__ void build_toeplitz(const double *__restrict__ hz, const double *__restrict__ left,
                               const double *__restrict__ right, int n, int ne, int npad,
                               int kpad, double scale, __half *__restrict__ thi,
                               __half *__restrict__ tlo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int k = blockIdx.z;
  if (i >= kpad) return;
  double v = 0.0;
  if (j < n && i < n) {
    if (i == 0) v = left[(size_t)k * n + j];
    else if (i == n - 1) v = right[(size_t)k * n + j];
    else {
      int d = j - i;
      if (d < 0) d += ne;
      v = hz[(size_t)k * ne + d];
    }
  }
  v *= scale;
  const __half h = __float2half_rn((float)v);
  const __half l = __float2half_rn((float)(v - (double)__half2float(h)));
  const size_t o = ((size_t)k * npad + j) * kpad + i;
  thi[o] = h;
  tlo[o] = l;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

// 2D fp16 tensor map: cols x rows with row pitch ld (elements), box 64 x box_rows.
int make_map(CUtensorMap *m, const void *ptr, size_t cols, size_t rows, size_t ld,
             uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) {
    set_error("tcfilter: cuTensorMapEncodeTiled unavailable");
    return TCB_ERR_CUDA;
  }
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * sizeof(__half))};
  cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void *>(ptr), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("tcfilter: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TCB_ERR_CUDA;
  }
  return TCB_OK;
}

void release(tcb_tcfilter *h) {
  cudaFree(h->thi);
  cudaFree(h->tlo);
  cudaFree(h->err);
  h->thi = h->tlo = nullptr;
  h->err = nullptr;
}

}  // namespace tcf
}  // namespace tcb

using namespace tcb;
using namespace tcb::tcf;

extern "C" int tcb_tcfilter_create(tcb_tcfilter **out, size_t nproj, size_t nz, size_t n,
                                   size_t nkern) {
  TCB_CHECK_ARG(out, "tcb_tcfilter_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 1 && nz >= 1 && nkern >= 1, "tcb_tcfilter_create: empty sizes");
  TCB_CHECK_ARG(n >= 64 && n % 8 == 0, "tcb_tcfilter_create: n must be >= 64 and a multiple of 8");
  TCB_CHECK_ARG(nproj * nz < (1ull << 31) && n <= 65536 && nkern <= 65536,
                "tcb_tcfilter_create: sizes too large");
  auto *h = new tcb_tcfilter{};
  h->nproj = nproj;
  h->nz = nz;
  h->n = n;
  h->nkern = nkern;
  h->npad = (int)((n + BN - 1) / BN * BN);
  h->kpad = (int)((n + BK - 1) / BK * BK);
  size_t tb = nkern * (size_t)h->npad * h->kpad * sizeof(__half);
  if (cudaMalloc(&h->thi, tb) != cudaSuccess || cudaMalloc(&h->tlo, tb) != cudaSuccess ||
      cudaMalloc(&h->err, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    release(h);
    delete h;
    set_error("tcb_tcfilter_create: out of device memory (%zu bytes of operator)", 2 * tb);
    return TCB_ERR_OUT_OF_MEMORY;
  }
  if (cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess) {
    release(h);
    delete h;
    set_error("tcb_tcfilter_create: cudaMemset failed");
    return TCB_ERR_CUDA;
  }
  static std::once_flag attr_once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once, [] {
    attr_err = cudaFuncSetAttribute(tcf_gemm<OUT_ROWS>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (attr_err == cudaSuccess)
      attr_err = cudaFuncSetAttribute(tcf_gemm<OUT_PAIRS>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  });
  if (attr_err != cudaSuccess) {
    release(h);
    delete h;
    set_error("tcb_tcfilter_create: cudaFuncSetAttribute failed: %s",
              cudaGetErrorString(attr_err));
    return TCB_ERR_CUDA;
  }
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_tcfilter_set_kernels(tcb_tcfilter *h, const double *hz, size_t ne,
                                        size_t pad, void *stream) {
  TCB_CHECK_ARG(h && hz, "tcb_tcfilter_set_kernels: null pointer");
  TCB_CHECK_ARG(h->thi, "tcb_tcfilter_set_kernels: handle was freed");
  const size_t n = h->n, nk = h->nkern;
  TCB_CHECK_ARG(ne >= n && pad + n <= ne, "tcb_tcfilter_set_kernels: need pad + n <= ne");
  TCB_CHECK_ARG(ne < (1u << 30), "tcb_tcfilter_set_kernels: ne too large");
  // Folded edge columns by prefix sums over two periods (float64, host).
  std::vector<double> left(nk * n), right(nk * n), cs(2 * ne + 1);
  double amax = 0.0;
  for (size_t k = 0; k < nk; k++) {
    const double *hk = hz + k * ne;
    // cs[t] = sum_{u=-ne}^{t-ne-1} hk[u mod ne]
    cs[0] = 0.0;
    for (size_t t = 0; t < 2 * ne; t++) cs[t + 1] = cs[t] + hk[t % ne];
    auto S = [&](long long a, long long b) {  // sum_{d=a}^{b} hk[d mod ne], -ne <= a
      return cs[(size_t)(b + 1 + (long long)ne)] - cs[(size_t)(a + (long long)ne)];
    };
    for (size_t j = 0; j < n; j++) {
      double l = S((long long)j, (long long)(j + pad));
      double r = S((long long)j + (long long)pad - (long long)ne + 1,
                   (long long)j - (long long)n + 1);
      left[k * n + j] = l;
      right[k * n + j] = r;
      amax = std::fmax(amax, std::fmax(std::fabs(l), std::fabs(r)));
    }
    for (size_t d = 0; d < ne; d++) amax = std::fmax(amax, std::fabs(hk[d]));
  }
  TCB_CHECK_ARG(amax > 0.0 && std::isfinite(amax), "tcb_tcfilter_set_kernels: degenerate kernel");
  // Largest power of two keeping every scaled entry <= 2^14 (fp16 max is 65504).
  int e = 0;
  std::frexp(amax, &e);  // amax in [2^(e-1), 2^e)
  const int sh = 14 - e;
  const double scale = std::ldexp(1.0, sh);
  cudaStream_t s = (cudaStream_t)stream;
  double *dhz = nullptr, *dl = nullptr, *dr = nullptr;
  int st = TCB_OK;
  if (cudaMalloc(&dhz, nk * ne * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&dl, nk * n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&dr, nk * n * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    set_error("tcb_tcfilter_set_kernels: out of device memory");
    st = TCB_ERR_OUT_OF_MEMORY;
  }
  if (st == TCB_OK) {
    cudaError_t ce =
        cudaMemcpyAsync(dhz, hz, nk * ne * sizeof(double), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(dl, left.data(), nk * n * sizeof(double), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(dr, right.data(), nk * n * sizeof(double), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) {
      dim3 grd(ceil_div((size_t)h->kpad, 256), (unsigned)h->npad, (unsigned)nk);
      build_toeplitz<<<grd, 256, 0, s>>>(dhz, dl, dr, (int)n, (int)ne, h->npad, h->kpad, scale,
                                         h->thi, h->tlo);
      count_launch();
      ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) {
      set_error("tcb_tcfilter_set_kernels: %s", cudaGetErrorString(ce));
      st = TCB_ERR_CUDA;
    }
  }
  cudaFree(dhz);
  cudaFree(dl);
  cudaFree(dr);
  if (st == TCB_OK) {
    h->inv_scale = (float)std::ldexp(1.0, -sh);
    h->ready = true;
  }
  return st;
}

extern "C" int tcb_tcfilter_apply(tcb_tcfilter *h, const void *x_hi, const void *x_lo,
                                  size_t lda, size_t nz, size_t kern0, void *out, int out_mode,
                                  size_t ldo, void *stream) {
  TCB_CHECK_ARG(h && x_hi && x_lo && out, "tcb_tcfilter_apply: null pointer");
  TCB_CHECK_ARG(h->thi, "tcb_tcfilter_apply: handle was freed");
  TCB_CHECK_ARG(h->ready, "tcb_tcfilter_apply: tcb_tcfilter_set_kernels was not called");
  TCB_CHECK_ARG(nz >= 1 && nz <= h->nz, "tcb_tcfilter_apply: nz out of range");
  TCB_CHECK_ARG(lda >= h->n && lda % 8 == 0,
                "tcb_tcfilter_apply: lda must be >= n and a multiple of 8");
  TCB_CHECK_ARG(((uintptr_t)x_hi & 15) == 0 && ((uintptr_t)x_lo & 15) == 0,
                "tcb_tcfilter_apply: operands must be 16-byte aligned");
  TCB_CHECK_ARG(out_mode == OUT_ROWS || out_mode == OUT_PAIRS,
                "tcb_tcfilter_apply: unknown out_mode %d", out_mode);
  TCB_CHECK_ARG(out_mode != OUT_ROWS || ldo >= h->n, "tcb_tcfilter_apply: ldo < n");
  TCB_CHECK_ARG(out_mode != OUT_PAIRS || nz % 2 == 0,
                "tcb_tcfilter_apply: paired output needs an even slice count");
  TCB_CHECK_ARG(h->nkern == 1 || kern0 + nz <= h->nkern,
                "tcb_tcfilter_apply: kernel range [kern0, kern0+nz) exceeds nkern");
  const size_t rows = nz * h->nproj;
  CUtensorMap ma_hi, ma_lo, mb_hi, mb_lo;
  int st;
  if ((st = make_map(&ma_hi, x_hi, h->n, rows, lda, BM)) != TCB_OK) return st;
  if ((st = make_map(&ma_lo, x_lo, h->n, rows, lda, BM)) != TCB_OK) return st;
  const size_t brows = h->nkern * (size_t)h->npad;
  if ((st = make_map(&mb_hi, h->thi, h->kpad, brows, h->kpad, BN)) != TCB_OK) return st;
  if ((st = make_map(&mb_lo, h->tlo, h->kpad, brows, h->kpad, BN)) != TCB_OK) return st;
  GemmArgs g;
  g.out = (float *)out;
  g.ldo = ldo;
  g.nproj = (int)h->nproj;
  g.nz = (int)nz;
  g.n = (int)h->n;
  g.zh = (int)(nz / 2);
  g.ptiles = (int)ceil_div(h->nproj, (size_t)BM);
  g.ntn = h->npad / BN;
  g.kblocks = h->kpad / BK;
  g.npad = h->npad;
  g.shared_kern = h->nkern == 1;
  g.kern0 = (int)kern0;
  g.inv_scale = h->inv_scale;
  g.err = h->err;
  const size_t ctas = nz * (size_t)g.ptiles * g.ntn;
  TCB_CHECK_ARG(ctas < (1ull << 31), "tcb_tcfilter_apply: too many tiles");
  cudaStream_t s = (cudaStream_t)stream;
  StageTimer tm("tc_filter", s);
  if (out_mode == OUT_ROWS)
    tcf_gemm<OUT_ROWS><<<(unsigned)ctas, 128, SMEM_BYTES, s>>>(ma_hi, ma_lo, mb_hi, mb_lo, g);
  else
    tcf_gemm<OUT_PAIRS><<<(unsigned)ctas, 128, SMEM_BYTES, s>>>(ma_hi, ma_lo, mb_hi, mb_lo, g);
  TCB_LAUNCH_CHECK();
  count_launch();
  return TCB_OK;
}

extern "C" int tcb_tcfilter_status(tcb_tcfilter *h, int *timed_out) {
  TCB_CHECK_ARG(h && timed_out, "tcb_tcfilter_status: null pointer");
  TCB_CHECK_ARG(h->err, "tcb_tcfilter_status: handle was freed");
  TCB_CUDA(cudaMemcpy(timed_out, h->err, sizeof(int), cudaMemcpyDeviceToHost));
  return TCB_OK;
}

extern "C" int tcb_tcfilter_destroy(tcb_tcfilter *h) {
  if (!h) return TCB_OK;
  release(h);
  delete h;
  return TCB_OK;
}
