// Single-distance phase retrieval of projections: Paganin, generalised
// Paganin and Farago filters (src/tomocupy/processing/retrieve_phase.py).
//
// The reference, per projection (_retrieve_phase, retrieve_phase.py:129-145):
// edge-pad the dy x dz image to Ny x Nz, complex fft2, multiply by the
// normalised real filter, ifft2, real part, crop.  Here:
//  * The filter F is real, so for a real image p,
//    real(ifft2(fft2(p) * F)) = ifft2(fft2(p) * Fe) with Fe(k) = (F(k) +
//    F(-k)) / 2 (the odd part of F maps the Hermitian spectrum of p to an
//    anti-Hermitian one, whose inverse transform is purely imaginary).  The
//    chain is therefore an R2C transform, a multiply by the half spectrum of
//    Fe (with the 1/(Ny Nz) normalisation folded in) and a C2R transform:
//    half the transform work and half the spectrum bytes of the reference's
//    C2C pair.  cuFFT runs the 2D transforms, batched over projections.
//  * Padding is index clamping in one kernel (the reference's four slice
//    assignments), cropping is a second kernel.
//  * Power-of-two padded sizes in [256, 8192] (the production case) run on
//    the library's own FFT instead, in three passes over two projections
//    packed as one complex image c = a + i b (Fe is real and even, so
//    ifft2(Fe fft2(c)) = a' + i b' with a', b' the filtered projections):
//    (1) per padded row: the padding (index clamping at load), the forward
//    FFT along the columns (conj(ifft(conj x))), stored in groups of 8
//    columns; (2) per column: the forward FFT along the rows, the product
//    with Fe, the inverse FFT, only the dy rows the crop keeps stored;
//    (3) per kept row: the inverse FFT along the columns and the crop into
//    the two projections in place.  The padded images and spectra never
//    exist in full: 3 passes instead of pad, R2C (2 passes), multiply, C2R
//    (2 passes) and crop.
//  * The filter is built once per geometry on the host with the reference's
//    float32 operation order (_reciprocal_grid, _paganin_filter_factor,
//    _farago_filter_factor, _paganin_filter_factorG, fftshift, / max).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "fft_pow2.cuh"

struct tcb_phase {
  size_t batch, dy, dz;  // projections per transform batch, image rows x columns
  size_t py, pz;         // padding of rows / columns (each side)
  size_t Ny, Nz;         // padded sizes
  cufftHandle fwd = 0, inv = 0;
  float *real = nullptr;   // [batch, Ny, Nz] padded images / filtered images
  float2 *spec = nullptr;  // [batch, Ny, Nz/2+1] spectra
  float *fe = nullptr;     // [Ny, Nz/2+1] even part of the normalised filter / (Ny Nz)
  // own-FFT chain (power-of-two Ny, Nz in [256, 8192]): packed pairs of projections
  bool own = false;
  float2 *t1 = nullptr;    // [pairs][Nz/8][Ny][8] row spectra, columns in groups of 8
  float2 *t2 = nullptr;    // [pairs][dy][Nz] filtered rows kept by the crop
  float2 *twy = nullptr, *twz = nullptr;  // twiddle tables of lengths Ny and Nz
};

namespace tcb {
namespace {

// Constants of retrieve_phase.py:45-48.
constexpr double PR_PLANCK = 6.58211928e-19;    // [keV*s]
constexpr double PR_LIGHT = 299792458e+2;        // [cm/s]
constexpr double PR_PI = 3.14159265359;

double wavelength(double energy) { return 2 * PR_PI * PR_PLANCK * PR_LIGHT / energy; }

// _calc_pad_width (retrieve_phase.py:224-226), float64 like the reference.
size_t pad_width(size_t dim, double pixel_size, double wl, double dist) {
  const double pad_pix = std::ceil(PR_PI * wl * dist / (pixel_size * pixel_size));
  const double p2 = std::pow(2.0, std::ceil(std::log2((double)dim + pad_pix)));
  return (size_t)(long long)((p2 - (double)dim) * 0.5);
}

// _reciprocal_coord (retrieve_phase.py:285-305): float32 arange(-n, N, 2) *
// float32(0.5 / (n * pixel_size)), n = N - 1.
std::vector<float> reciprocal_coord(double pixel_size, size_t num) {
  const long long n = (long long)num - 1;
  const float s = (float)(0.5 / ((double)n * pixel_size));
  std::vector<float> rc(num);
  for (size_t i = 0; i < num; i++) rc[i] = (float)(-n + 2 * (long long)i) * s;
  return rc;
}

// The reference's filter on the Ny x Nz grid (rows x columns), float32,
// before fftshift.
std::vector<float> filter_factor(int method, size_t Ny, size_t Nz, double pixel_size,
                                 double dist, double energy, double alpha, double db,
                                 double W) {
  const double wl = wavelength(energy);
  std::vector<float> f(Ny * Nz);
  if (method == TCB_PHASE_GPAGANIN) {
    // _reciprocal_gridG (retrieve_phase.py:261-282): cos(rc * 2 * PI * ps)
    // per axis, summed; _paganin_filter_factorG (:214-221)
    std::vector<float> cx = reciprocal_coord(pixel_size, Ny), cy = reciprocal_coord(pixel_size, Nz);
    const float two = 2.0f, pi = (float)PR_PI, ps = (float)pixel_size;
    for (auto &v : cx) v = std::cos(((v * two) * pi) * ps);
    for (auto &v : cy) v = std::cos(((v * two) * pi) * ps);
    const double aph = db * (dist * wl) / (4 * PR_PI);
    const float c = (float)(2 * aph / (W * W));
    for (size_t i = 0; i < Ny; i++)
      for (size_t j = 0; j < Nz; j++) {
        const float kf = cy[j] + cx[i];
        f[i * Nz + j] = 1.0f / (1.0f - c * (kf - 2.0f));
      }
    return f;
  }
  // _reciprocal_grid (retrieve_phase.py:229-258): squared coordinates,
  // meshgrid(indy, indx) summed as indy[j] + indx[i]
  std::vector<float> ix = reciprocal_coord(pixel_size, Ny), iy = reciprocal_coord(pixel_size, Nz);
  for (auto &v : ix) v = v * v;
  for (auto &v : iy) v = v * v;
  if (method == TCB_PHASE_PAGANIN) {
    // 1 / (wavelength * dist * w2 / (4 * PI) + alpha) (:209-210)
    const float a = (float)(wl * dist), d = (float)(4 * PR_PI), al = (float)alpha;
    for (size_t i = 0; i < Ny; i++)
      for (size_t j = 0; j < Nz; j++) {
        const float w2 = iy[j] + ix[i];
        f[i * Nz + j] = 1.0f / (a * w2 / d + al);
      }
  } else {
    // 1 / (cos(PI*wl*dist*w2) + db*sin(PI*wl*dist*w2)) (:212-213)
    const float a = (float)(PR_PI * wl * dist), b = (float)db;
    for (size_t i = 0; i < Ny; i++)
      for (size_t j = 0; j < Nz; j++) {
        const float t = a * (iy[j] + ix[i]);
        f[i * Nz + j] = 1.0f / (std::cos(t) + b * std::sin(t));
      }
  }
  return f;
}

// Index of padded position i on an axis with padding p and data length d:
// the reference's edge replication, prj[:p] = prj[p] and prj[-p:] =
// prj[-p-1] (retrieve_phase.py:138-141).  With p = 0 the second assignment
// is prj[0:] = prj[-1], which sets the whole axis to its last entry; kept.
__device__ __forceinline__ int pad_src(int i, int p, int d) {
  if (p == 0) return d - 1;
  return min(max(i - p, 0), d - 1);
}

// PR_ROWS rows per thread: the loads of one thread are independent, so
// each thread keeps PR_ROWS requests in flight (one row per thread left
// the kernel latency-bound at ~1.8 TB/s); every warp access stays a run of
// 32 consecutive floats.
constexpr int PR_ROWS = 4;

__global__ void phase_pad(float *__restrict__ out, const float *__restrict__ in, int dy, int dz,
                          int py, int pz, int Ny, int Nz) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * PR_ROWS;
  const size_t b = blockIdx.z;
  if (j >= Nz) return;
  const int sj = pad_src(j, pz, dz);
  float v[PR_ROWS];
#pragma unroll
  for (int r = 0; r < PR_ROWS; r++)
    if (i0 + r < Ny) v[r] = __ldg(in + (b * dy + pad_src(i0 + r, py, dy)) * dz + sj);
#pragma unroll
  for (int r = 0; r < PR_ROWS; r++)
    if (i0 + r < Ny) out[(b * Ny + i0 + r) * Nz + j] = v[r];
}

// one row of the half spectrum per block row, PR_ROWS projections of the
// batch per thread (the filter entry is loaded once for all of them)
__global__ void phase_mul(float2 *__restrict__ spec, const float *__restrict__ fe, int nc,
                          size_t plane, int nb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  const size_t e = (size_t)blockIdx.y * nc + k;  // entry within a spectrum
  const float w = __ldg(fe + e);
  const int b0 = blockIdx.z * PR_ROWS;
  float2 v[PR_ROWS];
#pragma unroll
  for (int r = 0; r < PR_ROWS; r++)
    if (b0 + r < nb) v[r] = spec[(size_t)(b0 + r) * plane + e];
#pragma unroll
  for (int r = 0; r < PR_ROWS; r++)
    if (b0 + r < nb) spec[(size_t)(b0 + r) * plane + e] = make_float2(v[r].x * w, v[r].y * w);
}

// Crop (retrieve_phase.py:143-144); with p = 0 nothing is cropped on that axis.
__global__ void phase_crop(float *__restrict__ out, const float *__restrict__ in, int dy, int dz,
                           int py, int pz, int Ny, int Nz) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * PR_ROWS;
  const size_t b = blockIdx.z;
  if (j >= dz) return;
  float v[PR_ROWS];
#pragma unroll
  for (int r = 0; r < PR_ROWS; r++)
    if (i0 + r < dy) v[r] = in[(b * Ny + i0 + r + py) * Nz + j + pz];
#pragma unroll
  for (int r = 0; r < PR_ROWS; r++)
    if (i0 + r < dy) out[(b * dy + i0 + r) * dz + j] = v[r];
}

// ---- own-FFT chain ------------------------------------------------------------
constexpr int PH_GW = 8;  // columns per group of the row-pass output

// Pass 1: padded row i of the pair (2q, 2q + 1): forward FFT along the
// columns of (a + i b), written to t1[q][j / 8][i][j % 8].
template <int N>
__global__ void __launch_bounds__(N / 16, (16384 / N < 16 ? 16384 / N : 16))
    ph_rows_fwd(const float *__restrict__ data, float2 *__restrict__ t1,
                const float2 *__restrict__ tw, int nb, int dy, int dz, int py, int pz, int Ny) {
  extern __shared__ float2 fsm[];
  const int i = blockIdx.x, q = blockIdx.y;
  const size_t img = (size_t)dy * dz;
  const float *a = data + (size_t)(2 * q) * img + (size_t)pad_src(i, py, dy) * dz;
  const float *b = 2 * q + 1 < nb ? a + img : nullptr;
  float2 *dst = t1 + (size_t)q * Ny * N + (size_t)i * PH_GW;
  // forward transform as conj(ifft(conj(x)))
  auto in = [a, b, pz, dz](int e) {
    const int j = pad_src(e, pz, dz);
    return make_float2(__ldg(a + j), b ? -__ldg(b + j) : 0.f);
  };
  auto out = [dst, Ny](int o, float2 v) {
    dst[(size_t)(o / PH_GW) * Ny * PH_GW + o % PH_GW] = make_float2(v.x, -v.y);
  };
  fftk::ifft<N>(fsm, threadIdx.x, tw, in, out);
}

// Pass 2: cpc adjacent columns j per block: forward FFT along the rows,
// product with the even filter Fe(k, j) (half table, Fe(k, j) = Fe(-k, -j)),
// inverse FFT, rows [py, py + dy) to t2[q][r][j].
template <int N>
__global__ void __launch_bounds__(1024)
    ph_cols(const float2 *__restrict__ t1, float2 *__restrict__ t2, const float *__restrict__ fe,
            const float2 *__restrict__ tw, int Nz, int dy, int py, int cpc) {
  extern __shared__ float2 fsm[];
  constexpr int SSTR = fftk::Plan<N>::PADDED + 4;
  const int c = threadIdx.x % cpc, tid = threadIdx.x / cpc;
  const int ncb = Nz / cpc;
  const int q = blockIdx.x / ncb, j = (blockIdx.x % ncb) * cpc + c;
  const int Nc = Nz / 2 + 1;
  const float2 *src = t1 + (size_t)q * N * Nz + (size_t)(j / PH_GW) * N * PH_GW + j % PH_GW;
  float2 *sm = fsm + c * SSTR;
  auto in1 = [src](int e) {
    const float2 v = __ldg(src + (size_t)e * PH_GW);
    return make_float2(v.x, -v.y);
  };
  auto out1 = [sm](int o, float2 v) { sm[fftk::pad16(o)] = make_float2(v.x, -v.y); };
  fftk::ifft<N, true>(sm, tid, tw, in1, out1);
  __syncthreads();
  {
    // times Fe(k, j) from the half table: column j, or row -k of column -j
    const bool neg = j >= Nc;
    const float *fcol = fe + (neg ? Nz - j : j);
#pragma unroll 4
    for (int k = tid; k < N; k += N / 16) {
      const float w = __ldg(fcol + (size_t)(neg ? (N - k) & (N - 1) : k) * Nc);
      float2 &x = sm[fftk::pad16(k)];
      x = make_float2(x.x * w, x.y * w);
    }
  }
  __syncthreads();
  float2 *dst = t2 + (size_t)q * dy * Nz + j;
  auto in2 = [sm](int e) { return sm[fftk::pad16(e)]; };
  auto out2 = [dst, py, dy, Nz](int o, float2 v) {
    const unsigned r = (unsigned)(o - py);
    if (r < (unsigned)dy) dst[(size_t)r * Nz] = v;
  };
  // the second transform reads the twiddles again instead of keeping the
  // first one's in registers (an opaque copy of the pointer)
  const float2 *tw2;
  asm volatile("mov.b64 %0, %1;" : "=l"(tw2) : "l"(tw));
  fftk::ifft<N>(sm, tid, tw2, in2, out2);
}

// Pass 3: kept row r: inverse FFT along the columns, columns [pz, pz + dz)
// written back to the two projections (real part to 2q, imaginary to 2q + 1).
template <int N>
__global__ void __launch_bounds__(N / 16, (16384 / N < 16 ? 16384 / N : 16))
    ph_rows_inv(const float2 *__restrict__ t2, float *__restrict__ data,
                const float2 *__restrict__ tw, int nb, int dy, int dz, int pz) {
  extern __shared__ float2 fsm[];
  const int r = blockIdx.x, q = blockIdx.y;
  const size_t img = (size_t)dy * dz;
  const float2 *src = t2 + ((size_t)q * dy + r) * N;
  float *a = data + (size_t)(2 * q) * img + (size_t)r * dz;
  float *b = 2 * q + 1 < nb ? a + img : nullptr;
  auto in = [src](int e) { return __ldg(src + e); };
  auto out = [a, b, pz, dz](int o, float2 v) {
    const unsigned j = (unsigned)(o - pz);
    if (j < (unsigned)dz) {
      a[j] = v.x;
      if (b) b[j] = v.y;
    }
  };
  fftk::ifft<N>(fsm, threadIdx.x, tw, in, out);
}

inline int ph_cpc(int N) { return std::min(16384 / N, 16); }
inline size_t ph_cols_smem(int N) { return (size_t)ph_cpc(N) * (N + N / 16 + 4) * sizeof(float2); }
inline size_t ph_rows_smem(int N) { return (size_t)(N + N / 16) * sizeof(float2); }

template <int N>
cudaError_t ph_attrs() {
  cudaError_t e = cudaFuncSetAttribute(ph_rows_fwd<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ph_rows_smem(N));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ph_rows_inv<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ph_rows_smem(N));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ph_cols<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ph_cols_smem(N));
  return e;
}

cudaError_t ph_attrs_for(int n) {
  switch (n) {
    case 256: return ph_attrs<256>();
    case 512: return ph_attrs<512>();
    case 1024: return ph_attrs<1024>();
    case 2048: return ph_attrs<2048>();
    case 4096: return ph_attrs<4096>();
    default: return ph_attrs<8192>();
  }
}

#define PH_DISPATCH(n, F)          \
  switch (n) {                     \
    case 256: F(256); break;       \
    case 512: F(512); break;       \
    case 1024: F(1024); break;     \
    case 2048: F(2048); break;     \
    case 4096: F(4096); break;     \
    default: F(8192); break;       \
  }

int ph_own_apply(tcb_phase *h, float *d, size_t b, cudaStream_t s) {
  const int Ny = (int)h->Ny, Nz = (int)h->Nz, dy = (int)h->dy, dz = (int)h->dz;
  const int py = (int)h->py, pz = (int)h->pz, nb = (int)b;
  const unsigned pairs = (unsigned)((b + 1) / 2);
  {
    StageTimer t("phase_rows_fwd", s);
#define PH_ROWS_FWD(N)                                                                   \
  ph_rows_fwd<N><<<dim3((unsigned)Ny, pairs), N / 16, ph_rows_smem(N), s>>>(             \
      d, h->t1, h->twz, nb, dy, dz, py, pz, Ny)
    PH_DISPATCH(Nz, PH_ROWS_FWD)
#undef PH_ROWS_FWD
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  {
    StageTimer t("phase_cols", s);
#define PH_COLS(N)                                                                       \
  ph_cols<N><<<(unsigned)(Nz / ph_cpc(N)) * pairs, ph_cpc(N) * (N / 16), ph_cols_smem(N), \
               s>>>(h->t1, h->t2, h->fe, h->twy, Nz, dy, py, ph_cpc(N))
    PH_DISPATCH(Ny, PH_COLS)
#undef PH_COLS
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  {
    StageTimer t("phase_rows_inv", s);
#define PH_ROWS_INV(N)                                                                   \
  ph_rows_inv<N><<<dim3((unsigned)dy, pairs), N / 16, ph_rows_smem(N), s>>>(             \
      h->t2, d, h->twz, nb, dy, dz, pz)
    PH_DISPATCH(Nz, PH_ROWS_INV)
#undef PH_ROWS_INV
    TCB_LAUNCH_CHECK();
    count_launch();
  }
  return TCB_OK;
}

bool pow2_in(size_t n) { return n >= 256 && n <= 8192 && (n & (n - 1)) == 0; }

void phase_release(tcb_phase *h) {
  if (h->fwd) cufftDestroy(h->fwd);
  if (h->inv) cufftDestroy(h->inv);
  cudaFree(h->real);
  cudaFree(h->spec);
  cudaFree(h->fe);
  cudaFree(h->t1);
  cudaFree(h->t2);
  cudaFree(h->twy);
  cudaFree(h->twz);
  h->fwd = h->inv = 0;
  h->real = h->fe = nullptr;
  h->spec = h->t1 = h->t2 = h->twy = h->twz = nullptr;
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_phase_pads(size_t dy, size_t dz, double pixel_size, double dist,
                              double energy, int pad, size_t *py, size_t *pz) {
  TCB_CHECK_ARG(py && pz, "tcb_phase_pads: null output");
  TCB_CHECK_ARG(dy >= 1 && dz >= 1, "tcb_phase_pads: empty image %zu x %zu", dy, dz);
  TCB_CHECK_ARG(pixel_size > 0 && energy > 0 && dist >= 0,
                "tcb_phase_pads: pixel_size and energy must be > 0, dist >= 0");
  *py = *pz = 0;
  if (pad) {
    const double wl = wavelength(energy);
    *py = pad_width(dy, pixel_size, wl, dist);
    *pz = pad_width(dz, pixel_size, wl, dist);
  }
  return TCB_OK;
}

extern "C" int tcb_phase_create(tcb_phase **out, size_t batch, size_t dy, size_t dz, int method,
                                double pixel_size, double dist, double energy, double alpha,
                                double db, double W, int pad) {
  TCB_CHECK_ARG(out, "tcb_phase_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(method == TCB_PHASE_PAGANIN || method == TCB_PHASE_GPAGANIN ||
                    method == TCB_PHASE_FARAGO,
                "tcb_phase_create: unknown method %d", method);
  TCB_CHECK_ARG(batch >= 1 && batch <= 65535, "tcb_phase_create: batch must be in [1, 65535]");
  TCB_CHECK_ARG(method != TCB_PHASE_GPAGANIN || W > 0, "tcb_phase_create: W must be > 0");
  size_t py = 0, pz = 0;
  int st = tcb_phase_pads(dy, dz, pixel_size, dist, energy, pad, &py, &pz);
  if (st != TCB_OK) return st;
  const size_t Ny = dy + 2 * py, Nz = dz + 2 * pz, Nc = Nz / 2 + 1;
  TCB_CHECK_ARG(Ny <= 65535 && Nz < (1u << 30) && Ny * Nz < (1ull << 31),
                "tcb_phase_create: padded image %zu x %zu too large", Ny, Nz);
  // the normalised filter, fftshifted, then its even part over the half spectrum
  std::vector<float> f = filter_factor(method, Ny, Nz, pixel_size, dist, energy, alpha, db, W);
  float fmax = -INFINITY;
  std::vector<float> sh(Ny * Nz);
  for (size_t i = 0; i < Ny; i++)
    for (size_t j = 0; j < Nz; j++) {
      // fftshift: output[i][j] = input[(i + Ny/2) % Ny][(j + Nz/2) % Nz]... with the
      // reference's convention (numpy fftshift shifts by floor(N/2))
      const float v = f[((i + Ny - Ny / 2) % Ny) * Nz + (j + Nz - Nz / 2) % Nz];
      sh[i * Nz + j] = v;
      fmax = std::max(fmax, v);
    }
  TCB_CHECK_ARG(std::isfinite(fmax) && fmax != 0.f,
                "tcb_phase_create: filter maximum %g is not finite and nonzero", (double)fmax);
  const float inv_n = (float)(1.0 / ((double)Ny * (double)Nz));
  std::vector<float> fe(Ny * Nc);
  for (size_t i = 0; i < Ny; i++)
    for (size_t j = 0; j < Nc; j++) {
      const float a = sh[i * Nz + j] / fmax;
      const float b = sh[((Ny - i) % Ny) * Nz + (Nz - j) % Nz] / fmax;
      fe[i * Nc + j] = 0.5f * (a + b) * inv_n;
    }

  tcb_phase *h = new tcb_phase();
  h->batch = batch;
  h->dy = dy;
  h->dz = dz;
  h->py = py;
  h->pz = pz;
  h->Ny = Ny;
  h->Nz = Nz;
  auto fail = [&](int code) {
    phase_release(h);
    delete h;
    return code;
  };
  h->own = pow2_in(Ny) && pow2_in(Nz) && std::getenv("TCB_PHASE_FFT") == nullptr;
  const size_t pairs = (batch + 1) / 2;
  bool okm = cudaMalloc(&h->fe, Ny * Nc * sizeof(float)) == cudaSuccess;
  if (okm && h->own)
    okm = cudaMalloc(&h->t1, pairs * Ny * Nz * sizeof(float2)) == cudaSuccess &&
          cudaMalloc(&h->t2, pairs * dy * Nz * sizeof(float2)) == cudaSuccess &&
          cudaMalloc(&h->twy, 2 * Ny * sizeof(float2)) == cudaSuccess &&
          cudaMalloc(&h->twz, 2 * Nz * sizeof(float2)) == cudaSuccess;
  else if (okm)
    okm = cudaMalloc(&h->real, batch * Ny * Nz * sizeof(float)) == cudaSuccess &&
          cudaMalloc(&h->spec, batch * Ny * Nc * sizeof(float2)) == cudaSuccess;
  if (!okm) {
    cudaGetLastError();
    set_error("tcb_phase_create: out of device memory (batch %zu of %zu x %zu)", batch, Ny, Nz);
    return fail(TCB_ERR_OUT_OF_MEMORY);
  }
  cudaError_t e = cudaMemcpy(h->fe, fe.data(), fe.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && h->own) {
    const std::vector<float2> ty = fftk::twiddle_table((int)Ny), tz = fftk::twiddle_table((int)Nz);
    if (ty.size() > 2 * Ny || tz.size() > 2 * Nz) {
      set_error("tcb_phase_create: twiddle table larger than its buffer");
      return fail(TCB_ERR_CUDA);
    }
    e = cudaMemcpy(h->twy, ty.data(), ty.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(h->twz, tz.data(), tz.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = ph_attrs_for((int)Ny);
    if (e == cudaSuccess) e = ph_attrs_for((int)Nz);
  }
  if (e != cudaSuccess) {
    set_error("tcb_phase_create: setup failed: %s", cudaGetErrorString(e));
    return fail(TCB_ERR_CUDA);
  }
  if (h->own) {
    *out = h;
    return TCB_OK;
  }
  int dims[2] = {(int)Ny, (int)Nz};
  cufftResult r = cufftPlanMany(&h->fwd, 2, dims, nullptr, 1, (int)(Ny * Nz), nullptr, 1,
                                (int)(Ny * Nc), CUFFT_R2C, (int)batch);
  if (r == CUFFT_SUCCESS)
    r = cufftPlanMany(&h->inv, 2, dims, nullptr, 1, (int)(Ny * Nc), nullptr, 1, (int)(Ny * Nz),
                      CUFFT_C2R, (int)batch);
  if (r != CUFFT_SUCCESS) {
    set_error("tcb_phase_create: cufftPlanMany failed: %d", (int)r);
    return fail(r == CUFFT_ALLOC_FAILED ? TCB_ERR_OUT_OF_MEMORY : TCB_ERR_CUFFT);
  }
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_phase_sizes(tcb_phase *h, size_t *py, size_t *pz) {
  TCB_CHECK_ARG(h && py && pz, "tcb_phase_sizes: null pointer");
  *py = h->py;
  *pz = h->pz;
  return TCB_OK;
}

extern "C" int tcb_phase_apply(tcb_phase *h, float *data, size_t nproj, void *stream) {
  TCB_CHECK_ARG(h, "tcb_phase_apply: null handle");
  TCB_CHECK_ARG(h->real || h->t1, "tcb_phase_apply: handle was freed");
  TCB_CHECK_ARG(data || nproj == 0, "tcb_phase_apply: null data");
  cudaStream_t s = (cudaStream_t)stream;
  if (h->own) {
    for (size_t p0 = 0; p0 < nproj; p0 += h->batch) {
      const int st = ph_own_apply(h, data + p0 * h->dy * h->dz, std::min(h->batch, nproj - p0), s);
      if (st != TCB_OK) return st;
    }
    return TCB_OK;
  }
  TCB_CUFFT(cufftSetStream(h->fwd, s));
  TCB_CUFFT(cufftSetStream(h->inv, s));
  const size_t Nc = h->Nz / 2 + 1, plane = h->Ny * Nc;
  for (size_t p0 = 0; p0 < nproj; p0 += h->batch) {
    const size_t b = std::min(h->batch, nproj - p0);
    float *d = data + p0 * h->dy * h->dz;
    {
      StageTimer t("phase_pad", s);
      phase_pad<<<dim3(ceil_div(h->Nz, 256), ceil_div(h->Ny, PR_ROWS), (unsigned)b), 256, 0, s>>>(
          h->real, d, (int)h->dy, (int)h->dz, (int)h->py, (int)h->pz, (int)h->Ny, (int)h->Nz);
      TCB_LAUNCH_CHECK();
      count_launch();
    }
    // a partial last batch runs the full-batch plan on stale padded images
    // beyond b; only the first b are cropped back
    {
      StageTimer t("phase_r2c", s);
      TCB_CUFFT(cufftExecR2C(h->fwd, h->real, (cufftComplex *)h->spec));
    }
    {
      StageTimer t("phase_mul", s);
      phase_mul<<<dim3(ceil_div(Nc, 256), (unsigned)h->Ny, ceil_div(b, PR_ROWS)), 256, 0, s>>>(
          h->spec, h->fe, (int)Nc, plane, (int)b);
      TCB_LAUNCH_CHECK();
      count_launch();
    }
    {
      StageTimer t("phase_c2r", s);
      TCB_CUFFT(cufftExecC2R(h->inv, (cufftComplex *)h->spec, h->real));
    }
    {
      StageTimer t("phase_crop", s);
      phase_crop<<<dim3(ceil_div(h->dz, 256), ceil_div(h->dy, PR_ROWS), (unsigned)b), 256, 0, s>>>(
          d, h->real, (int)h->dy, (int)h->dz, (int)h->py, (int)h->pz, (int)h->Ny, (int)h->Nz);
      TCB_LAUNCH_CHECK();
      count_launch();
    }
  }
  return TCB_OK;
}

extern "C" int tcb_phase_destroy(tcb_phase *h) {
  if (!h) return TCB_OK;
  phase_release(h);
  delete h;
  return TCB_OK;
}
