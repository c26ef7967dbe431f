// Vo's all-stripe ring removal (remove_all_stripe, src/tomocupy/processing/
// remove_stripe.py:311-498; N. T. Vo et al., Opt. Express 26 (2018), algorithms
// 3-6) on a sinogram chunk tomo[p][z][x] (nproj angles, nz rows, ni columns),
// in place:
//  1. dead stripes (_rs_dead3): per column the total variation along the
//     angles against a 10-angle moving mean; columns whose variation stands
//     out from its median over la_size columns are flagged (stripe
//     detection, one-column dilation, the two outer columns on each side
//     never flagged) and replaced by linear interpolation between their
//     nearest unflagged neighbours;
//  2. large stripes (_rs_large3): every column sorted along the angles, the
//     sorted values smoothed by a median over la_size columns, columns whose
//     mean sorted value differs from the smoothed one flagged; all columns
//     divided by the ratio, flagged columns replaced by the smoothed values
//     put back in angle order;
//  3. small and medium stripes (_rs_sort3): the sorted values smoothed by a
//     median over sm_size columns and put back in angle order.
// B200 design: one CTA sorts one column (64-bit keys: the float's order bits
// and the angle, so equal values keep their angle order, as CuPy's stable
// argsort); the median along the detector is a sliding window per thread
// (a sorted window in shared memory, one replacement per output column, the
// threads of a warp on consecutive ranks so every read is coalesced); the
// per-row statistics (stripe detection) are one CTA per row.  Float32
// reductions add in another order than the reference's, so results agree
// to float rounding; the sorts, medians and interpolation weights are exact.
#include <algorithm>
#include <cmath>

#include "common.cuh"

struct tcb_stripe_vo {
  size_t nproj, nz, ni;
  float snr;
  int la, sm;
  float *tt = nullptr;       // [nz][ni][nproj] the chunk with contiguous columns
  float *srt = nullptr;      // [nz][ni][nproj] values sorted along the angles
  int *ids = nullptr;        // [nz][ni][nproj] angle of each sorted value
  float *smooth = nullptr;   // [nz][ni][nproj]
  float *l1 = nullptr, *l2 = nullptr;  // [nz][ni] per-column statistics
  float *mask = nullptr;     // [nz][ni]
  float *fact = nullptr;     // [nz][ni]
  int2 *nbr = nullptr;       // [nz][ni] nearest unflagged columns (left, right)
};

namespace tcb {
namespace {

constexpr int VO_MED_T = 128;  // threads per median block
constexpr int VO_RUN = 128;    // output columns per median thread
constexpr int VO_MAXW = 127;   // largest median window

__device__ __forceinline__ int reflect_idx(int i, int n) {
  // scipy.ndimage mode 'reflect' (d c b a | a b c d | d c b a)
  const int p = 2 * n;
  int m = i % p;
  if (m < 0) m += p;
  return m >= n ? p - 1 - m : m;
}

// Total order of floats as unsigned integers (negative values reversed).
__device__ __forceinline__ uint32_t fkey(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float fdecode(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// Compare-exchange of key a (index i) with its partner b: the lower index
// keeps the smaller key in an ascending run (i & k == 0), the larger in a
// descending one.
__device__ __forceinline__ unsigned long long bitonic_keep(unsigned long long a,
                                                           unsigned long long b, int i, int j,
                                                           int k) {
  const bool up = (i & k) == 0, lower = (i & j) == 0;
  return (lower == up) ? (a < b ? a : b) : (a < b ? b : a);
}

// The exchanges at distance J < E among a thread's own keys.
template <int E, int J>
__device__ __forceinline__ void in_thread(unsigned long long (&v)[E], int t, int k) {
#pragma unroll
  for (int e = 0; e < E; e++) {
    if ((e & J) == 0) {
      const int i = t * E + e;
      const unsigned long long a = v[e], b = v[e | J];
      const bool up = (i & k) == 0;
      v[e] = (a < b) == up ? a : b;
      v[e | J] = (a < b) == up ? b : a;
    }
  }
}

// One CTA per column (z, x): the nproj values sorted ascending, ties in
// angle order; srt/ids [(z * ni + x) * nproj + r].  Bitonic sort of p2 =
// E * blockDim 64-bit keys (order bits of the value, angle): thread t holds
// keys t*E .. t*E + E - 1 in registers; exchanges at distance j < E stay in
// the thread, E <= j < 32 E go through warp shuffles, only the longer ones
// through shared memory.  The sorted values are decoded from the keys.
template <int E>
__global__ void vo_sort_cols(const float *__restrict__ tomo, size_t pstride, size_t zstride,
                             size_t xstride, int nproj, int ni, int p2, float *__restrict__ srt,
                             int *__restrict__ ids) {
  extern __shared__ unsigned long long key[];
  const int x = blockIdx.x, z = blockIdx.y, t = threadIdx.x;
  const float *col = tomo + (size_t)z * zstride + (size_t)x * xstride;
  unsigned long long v[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int r = t * E + e;
    const uint32_t k = r < nproj ? fkey(col[(size_t)r * pstride]) : 0xFFFFFFFFu;
    v[e] = ((unsigned long long)k << 32) | (unsigned)r;
  }
  for (int k = 2; k <= p2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j < E) {
        if (j == 1) in_thread<E, 1>(v, t, k);
        else if (j == 2) in_thread<E, 2>(v, t, k);
        else if (E > 4) in_thread<E, (E > 4 ? 4 : 1)>(v, t, k);
      } else if (j < 32 * E) {
        const int lm = j / E;  // partner lane
#pragma unroll
        for (int e = 0; e < E; e++) {
          const unsigned long long b = __shfl_xor_sync(0xffffffffu, v[e], lm);
          v[e] = bitonic_keep(v[e], b, t * E + e, j, k);
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; e++) key[t * E + e] = v[e];
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int i = t * E + e;
          v[e] = bitonic_keep(v[e], key[i ^ j], i, j, k);
        }
        __syncthreads();
      }
    }
  float *so = srt + ((size_t)z * ni + x) * nproj;
  int *io = ids + ((size_t)z * ni + x) * nproj;
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int r = t * E + e;
    if (r < nproj) {
      so[r] = fdecode((uint32_t)(v[e] >> 32));
      io[r] = (int)(v[e] & 0xFFFFFFFFu);
    }
  }
}

// keys per thread and threads for a column of p2 (power of two) keys
inline int sort_e(int p2) { return p2 <= 4096 ? 4 : 8; }

// Median over w (odd) columns, reflect mode, of in[(z * ni + x) * R + r] for
// every (z, x, r): each thread slides a sorted window along a run of VO_RUN
// columns of one (z, r) (window kept interleaved in shared memory).
__global__ void __launch_bounds__(VO_MED_T)
    vo_median_x(const float *__restrict__ in, float *__restrict__ out, int nz, int ni, int R,
                int w) {
  extern __shared__ float win[];  // win[j * VO_MED_T + t]
  const int t = threadIdx.x;
  const long long g = (long long)blockIdx.x * VO_MED_T + t;
  const int nrun = (ni + VO_RUN - 1) / VO_RUN;
  if (g >= (long long)nz * nrun * R) return;
  const int r = (int)(g % R);
  const long long q = g / R;
  const int run = (int)(q % nrun), z = (int)(q / nrun);
  const int x0 = run * VO_RUN, x1 = min(ni, x0 + VO_RUN), h = w / 2;
  auto val = [&](int x) { return in[((size_t)z * ni + reflect_idx(x, ni)) * R + r]; };
  auto W = [&](int i) -> float & { return win[i * VO_MED_T + t]; };
  for (int j = 0; j < w; j++) {  // insertion sort of the first window
    const float v = val(x0 - h + j);
    int i = j;
    while (i > 0 && W(i - 1) > v) {
      W(i) = W(i - 1);
      i--;
    }
    W(i) = v;
  }
  out[((size_t)z * ni + x0) * R + r] = W(h);
  for (int x = x0 + 1; x < x1; x++) {
    const float vo = val(x - h - 1), vn = val(x + h);
    int lo = 0, hi = w - 1;  // first position holding a value >= vo (vo is present)
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (W(mid) < vo) lo = mid + 1; else hi = mid;
    }
    int i = lo;
    W(i) = vn;
    while (i + 1 < w && W(i + 1) < W(i)) {
      const float a = W(i);
      W(i) = W(i + 1);
      W(i + 1) = a;
      i++;
    }
    while (i > 0 && W(i - 1) > W(i)) {
      const float a = W(i);
      W(i) = W(i - 1);
      W(i - 1) = a;
      i--;
    }
    out[((size_t)z * ni + x) * R + r] = W(h);
  }
}

// _rs_dead3's column variation: diff[z][x] = sum_p |tomo - uniform_filter1d(
// tomo, 10, axis=0)| (reflect mode; window p-5 .. p+4, a float64 running sum
// divided by 10 and rounded, as scipy's filter), accumulated in float32 in
// angle order.  One thread per column.
__global__ void vo_dead_diff(const float *__restrict__ tomo, size_t pstride, size_t zstride,
                             int nproj, int nz, int ni, float *__restrict__ diff) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
  if (x >= ni) return;
  const float *col = tomo + (size_t)z * zstride + x;
  auto v = [&](int p) { return (double)col[(size_t)reflect_idx(p, nproj) * pstride]; };
  double run = 0.0;
  for (int p = -5; p <= 4; p++) run += v(p);
  float acc = 0.f;
  for (int p = 0; p < nproj; p++) {
    const float m = (float)(run / 10.0);
    acc += fabsf(col[(size_t)p * pstride] - m);
    run += v(p + 5) - v(p - 5);
  }
  diff[(size_t)z * ni + x] = acc;
}

// Mean over ranks [nd, nproj - nd) of sorted and smoothed columns -> l1, l2.
// One warp per column.
__global__ void vo_rank_means(const float *__restrict__ srt, const float *__restrict__ sm,
                              int nproj, int ncol, int nd, float *__restrict__ l1,
                              float *__restrict__ l2) {
  const int wc = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (wc >= ncol) return;
  const float *a = srt + (size_t)wc * nproj, *b = sm + (size_t)wc * nproj;
  float s1 = 0.f, s2 = 0.f;
  for (int r = nd + lane; r < nproj - nd; r += 32) {
    s1 += a[r];
    s2 += b[r];
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    const float cnt = (float)(nproj - 2 * nd);
    l1[wc] = s1 / cnt;
    l2[wc] = s2 / cnt;
  }
}

// _detect_stripe_batch + binary_dilation((1, 3)) on fact[z] = num[z] / den[z]
// (remove_stripe.py:346-370): one CTA per row.  dead != 0 also clears the two
// outer columns on each side and writes the nearest unflagged columns of
// every flagged one.  Line fit in float32 as the reference (its sums in
// float64 here).
__global__ void vo_detect(const float *__restrict__ num, const float *__restrict__ den, int ni,
                          int p2, float snr, int dead, float *__restrict__ fact,
                          float *__restrict__ mask, int2 *__restrict__ nbr) {
  extern __shared__ unsigned char vsm[];
  float *f = reinterpret_cast<float *>(vsm);               // [ni] ratio
  uint32_t *k = reinterpret_cast<uint32_t *>(f + ni);      // [p2] sort keys
  float *m = reinterpret_cast<float *>(k + p2);            // [ni] raw mask
  __shared__ double red[2][32];
  __shared__ float stat[4];
  const int z = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  for (int x = tid; x < ni; x += nt) {
    const float v = num[(size_t)z * ni + x] / den[(size_t)z * ni + x];
    f[x] = v;
    fact[(size_t)z * ni + x] = v;
  }
  for (int i = tid; i < p2; i += nt) k[i] = i < ni ? ~fkey(f[i]) : 0xFFFFFFFFu;  // descending
  __syncthreads();
  for (int kk = 2; kk <= p2; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < p2; i += nt) {
        const int l = i ^ j;
        if (l > i) {
          const uint32_t a = k[i], b = k[l];
          if ((a > b) == ((i & kk) == 0)) {
            k[i] = b;
            k[l] = a;
          }
        }
      }
      __syncthreads();
    }
  auto sval = [&](int i) {  // i-th largest value
    const uint32_t u = ~k[i];
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
  };
  const int nd = (int)(0.25 * ni);
  const int a = nd, b = ni - nd - 1;  // listsorted[:, nd:-nd-1]
  double sy = 0.0, sxy = 0.0;
  for (int i = a + tid; i < b; i += nt) {
    const double y = sval(i);
    sy += y;
    sxy += y * (double)i;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
    sxy += __shfl_xor_sync(0xffffffffu, sxy, o);
  }
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = sy;
    red[1][tid >> 5] = sxy;
  }
  __syncthreads();
  if (tid == 0) {
    double ty = 0.0, txy = 0.0;
    for (int w = 0; w < (nt + 31) / 32; w++) {
      ty += red[0][w];
      txy += red[1][w];
    }
    const int n = b - a;
    double sx = 0.0, sxx = 0.0;
    for (int i = a; i < b; i++) {
      sx += i;
      sxx += (double)i * i;
    }
    const float xm = (float)(sx / n), ym = (float)(ty / n);
    const float Sxy = (float)txy - (float)n * ym * xm;
    const float Sxx = (float)(sxx - (double)n * xm * xm);
    const float slope = Sxy / Sxx;
    const float icpt = ym - slope * xm;
    const float numt1 = icpt + slope * (float)(ni - 1);
    const float noise = fmaxf(fabsf(numt1 - icpt), 1e-6f);
    const float val1 = fabsf(sval(0) - icpt) / noise;
    const float val2 = fabsf(sval(ni - 1) - numt1) / noise;
    stat[0] = val1 >= snr ? icpt + noise * snr * 0.5f : INFINITY;   // upper threshold
    stat[1] = val2 >= snr ? numt1 - noise * snr * 0.5f : -INFINITY; // lower threshold
  }
  __syncthreads();
  const float up = stat[0], lo = stat[1];
  for (int x = tid; x < ni; x += nt) m[x] = (f[x] > up || f[x] <= lo) ? 1.f : 0.f;
  __syncthreads();
  for (int x = tid; x < ni; x += nt) {
    float v = m[x];
    if (x > 0) v = fmaxf(v, m[x - 1]);
    if (x + 1 < ni) v = fmaxf(v, m[x + 1]);
    if (dead && (x < 2 || x >= ni - 2)) v = 0.f;
    mask[(size_t)z * ni + x] = v;
  }
  if (!dead) return;
  __syncthreads();
  for (int x = tid; x < ni; x += nt) m[x] = mask[(size_t)z * ni + x];
  __syncthreads();
  for (int x = tid; x < ni; x += nt) {
    int l = x, r = x;
    if (m[x] > 0.f) {
      while (l > 0 && m[l] > 0.f) l--;
      while (r < ni - 1 && m[r] > 0.f) r++;
    }
    nbr[(size_t)z * ni + x] = make_int2(l, r);
  }
}

// Flagged dead columns: linear interpolation between the nearest unflagged
// columns, tl + (x - xl) * (tr - tl) / (xr - xl) with tr - tl in float32 and
// the rest in float64 (the reference's NumPy/CuPy type promotion).
__global__ void vo_dead_interp(float *__restrict__ tomo, size_t pstride, size_t zstride, int nproj,
                               int ni, const float *__restrict__ mask,
                               const int2 *__restrict__ nbr) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
  if (x >= ni || mask[(size_t)z * ni + x] <= 0.f) return;
  const int2 lr = nbr[(size_t)z * ni + x];
  float *row = tomo + (size_t)z * zstride;
  for (int p = blockIdx.z; p < nproj; p += gridDim.z) {
    const float tl = row[(size_t)p * pstride + lr.x], tr = row[(size_t)p * pstride + lr.y];
    const double d = (double)(x - lr.x) * (double)(tr - tl) / (double)(lr.y - lr.x);
    row[(size_t)p * pstride + x] = (float)((double)tl + d);
  }
}

// tt[z][x][ids[r]] = vals[z][x][r] for the columns whose mask is set (or all).
__global__ void vo_unsort(float *__restrict__ tt, int nproj, int ni,
                          const float *__restrict__ vals, const int *__restrict__ ids,
                          const float *__restrict__ mask) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int x = blockIdx.y, z = blockIdx.z;
  if (r >= nproj) return;
  if (mask && mask[(size_t)z * ni + x] <= 0.f) return;
  const size_t c = ((size_t)z * ni + x) * nproj;
  tt[c + ids[c + r]] = vals[c + r];
}

// tt[z][x][p] /= fact[z][x]
__global__ void vo_divide_t(float *__restrict__ tt, int nproj, size_t total,
                            const float *__restrict__ fact) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  tt[i] /= fact[i / nproj];
}

// [z][p][x] (strides pstride, zstride; x contiguous) <-> [z][x][p], 32 x 32
// shared-memory tiles; to_t: towards the column-contiguous layout.
__global__ void vo_transpose(float *__restrict__ tomo, size_t pstride, size_t zstride,
                             float *__restrict__ tt, int nproj, int ni, int to_t) {
  __shared__ float tile[32][33];
  const int z = blockIdx.z;
  const int p0 = blockIdx.y * 32, x0 = blockIdx.x * 32;
  float *row = tomo + (size_t)z * zstride;
  float *colt = tt + (size_t)z * ni * nproj;
  if (to_t) {
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
      const int p = p0 + k, x = x0 + threadIdx.x;
      if (p < nproj && x < ni) tile[k][threadIdx.x] = row[(size_t)p * pstride + x];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
      const int x = x0 + k, p = p0 + threadIdx.x;
      if (p < nproj && x < ni) colt[(size_t)x * nproj + p] = tile[threadIdx.x][k];
    }
  } else {
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
      const int x = x0 + k, p = p0 + threadIdx.x;
      if (p < nproj && x < ni) tile[threadIdx.x][k] = colt[(size_t)x * nproj + p];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
      const int p = p0 + k, x = x0 + threadIdx.x;
      if (p < nproj && x < ni) row[(size_t)p * pstride + x] = tile[k][threadIdx.x];
    }
  }
}

void vo_release(tcb_stripe_vo *h) {
  cudaFree(h->tt);
  h->tt = nullptr;
  cudaFree(h->srt);
  cudaFree(h->ids);
  cudaFree(h->smooth);
  cudaFree(h->l1);
  cudaFree(h->l2);
  cudaFree(h->mask);
  cudaFree(h->fact);
  cudaFree(h->nbr);
  h->srt = h->smooth = h->l1 = h->l2 = h->mask = h->fact = nullptr;
  h->ids = nullptr;
  h->nbr = nullptr;
}

int pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace
}  // namespace tcb

using namespace tcb;

extern "C" int tcb_stripe_vo_create(tcb_stripe_vo **out, size_t nproj, size_t nz, size_t ni,
                                    double snr, int la_size, int sm_size, int dim) {
  TCB_CHECK_ARG(out, "tcb_stripe_vo_create: null out");
  *out = nullptr;
  TCB_CHECK_ARG(nproj >= 12 && nproj <= 8192 && nz >= 1 && nz <= 65535 && ni >= 8 &&
                    ni <= 8192,
                "tcb_stripe_vo_create: sizes nproj=%zu (12..8192), nz=%zu, ni=%zu (8..8192)",
                nproj, nz, ni);
  TCB_CHECK_ARG(la_size >= 1 && la_size <= VO_MAXW && la_size % 2 == 1 && sm_size >= 1 &&
                    sm_size <= VO_MAXW && sm_size % 2 == 1,
                "tcb_stripe_vo_create: median windows must be odd and <= %d (got %d, %d)",
                VO_MAXW, la_size, sm_size);
  TCB_CHECK_ARG(dim == 1, "tcb_stripe_vo_create: only dim 1 (windows along the detector)");
  TCB_CHECK_ARG(std::isfinite(snr), "tcb_stripe_vo_create: bad snr");
  tcb_stripe_vo *h = new tcb_stripe_vo();
  h->nproj = nproj;
  h->nz = nz;
  h->ni = ni;
  h->snr = (float)snr;
  h->la = la_size;
  h->sm = sm_size;
  const size_t cols = nz * ni, vals = cols * nproj;
  if (cudaMalloc(&h->tt, vals * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->srt, vals * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->ids, vals * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&h->smooth, vals * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->l1, cols * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->l2, cols * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->mask, cols * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->fact, cols * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->nbr, cols * sizeof(int2)) != cudaSuccess) {
    cudaGetLastError();
    vo_release(h);
    delete h;
    set_error("tcb_stripe_vo_create: out of device memory");
    return TCB_ERR_OUT_OF_MEMORY;
  }
  const int sort_smem = std::max(pow2_at_least((int)nproj), 128) * 8;
  const int med_smem = VO_MAXW * VO_MED_T * 4;
  if (cudaFuncSetAttribute(vo_sort_cols<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           sort_smem) != cudaSuccess ||
      cudaFuncSetAttribute(vo_sort_cols<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           sort_smem) != cudaSuccess ||
      cudaFuncSetAttribute(vo_median_x, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           med_smem) != cudaSuccess ||
      cudaFuncSetAttribute(vo_detect, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(2 * ni * 4 + pow2_at_least((int)ni) * 4)) != cudaSuccess) {
    vo_release(h);
    delete h;
    set_error("tcb_stripe_vo_create: shared-memory attribute failed");
    return TCB_ERR_CUDA;
  }
  *out = h;
  return TCB_OK;
}

extern "C" int tcb_stripe_vo_apply(tcb_stripe_vo *h, float *tomo, size_t pstride,
                                   size_t zstride, void *stream) {
  TCB_CHECK_ARG(h && h->srt, "tcb_stripe_vo_apply: null or freed handle");
  TCB_CHECK_ARG(tomo, "tcb_stripe_vo_apply: null data");
  TCB_CHECK_ARG(zstride >= h->ni && pstride >= h->ni &&
                    (pstride >= (h->nz - 1) * zstride + h->ni ||
                     zstride >= (h->nproj - 1) * pstride + h->ni),
                "tcb_stripe_vo_apply: strides make rows overlap");
  cudaStream_t s = (cudaStream_t)stream;
  const int np = (int)h->nproj, nz = (int)h->nz, ni = (int)h->ni;
  // at least a full warp of threads (the shuffle stages)
  const int p2 = std::max(pow2_at_least(np), 128), n2 = pow2_at_least(ni);
  const dim3 cgrid(ceil_div(h->ni, 128), nz), pgrid(ceil_div(h->ni, 128), nz, 16);
  const int nd = (int)(0.5 * 0.1 * np);  // drop_ratio 0.1
  const int dsm = (int)(2 * h->ni * 4 + n2 * 4);
  // sorts read the column-contiguous copy tt
  auto sort_cols = [&]() {
    const size_t zs = (size_t)ni * np;
    if (sort_e(p2) == 4)
      vo_sort_cols<4><<<dim3(ni, nz), p2 / 4, (size_t)p2 * 8, s>>>(h->tt, 1, zs, np, np, ni, p2,
                                                                   h->srt, h->ids);
    else
      vo_sort_cols<8><<<dim3(ni, nz), p2 / 8, (size_t)p2 * 8, s>>>(h->tt, 1, zs, np, np, ni, p2,
                                                                   h->srt, h->ids);
  };
  const dim3 tgrid(ceil_div(h->ni, 32), ceil_div(h->nproj, 32), nz), tblk(32, 8);
  auto median = [&](const float *in, float *outp, int R, int w) {
    const int nrun = (ni + VO_RUN - 1) / VO_RUN;
    const long long thr = (long long)nz * nrun * R;
    vo_median_x<<<(unsigned)((thr + VO_MED_T - 1) / VO_MED_T), VO_MED_T,
                  (size_t)w * VO_MED_T * 4, s>>>(in, outp, nz, ni, R, w);
  };
  StageTimer t("stripe_vo", s);
  // 1. dead stripes
  {
    StageTimer st("stripe_vo_dead", s);
    vo_dead_diff<<<cgrid, 128, 0, s>>>(tomo, pstride, zstride, np, nz, ni, h->l1);
    median(h->l1, h->l2, 1, h->la);
    vo_detect<<<nz, 256, dsm, s>>>(h->l1, h->l2, ni, n2, h->snr, 1, h->fact, h->mask, h->nbr);
    vo_dead_interp<<<pgrid, 128, 0, s>>>(tomo, pstride, zstride, np, ni, h->mask, h->nbr);
    TCB_LAUNCH_CHECK();
  }
  // 2. large stripes (on the column-contiguous copy)
  {
    StageTimer st("stripe_vo_sort", s);
    vo_transpose<<<tgrid, tblk, 0, s>>>(tomo, pstride, zstride, h->tt, np, ni, 1);
    sort_cols();
  }
  {
    StageTimer st("stripe_vo_median", s);
    median(h->srt, h->smooth, np, h->la);
  }
  const size_t vals = (size_t)nz * ni * np;
  {
    StageTimer st("stripe_vo_large", s);
    vo_rank_means<<<ceil_div(h->nz * h->ni * 32, 256), 256, 0, s>>>(h->srt, h->smooth, np,
                                                                    nz * ni, nd, h->l1, h->l2);
    vo_detect<<<nz, 256, dsm, s>>>(h->l1, h->l2, ni, n2, h->snr, 0, h->fact, h->mask, h->nbr);
    vo_divide_t<<<ceil_div(vals, 256), 256, 0, s>>>(h->tt, np, vals, h->fact);
  }
  {
    StageTimer st("stripe_vo_unsort", s);
    vo_unsort<<<dim3(ceil_div(h->nproj, 128), ni, nz), 128, 0, s>>>(h->tt, np, ni, h->smooth,
                                                                    h->ids, h->mask);
  }
  TCB_LAUNCH_CHECK();
  // 3. small and medium stripes
  {
    StageTimer st("stripe_vo_sort", s);
    sort_cols();
  }
  {
    StageTimer st("stripe_vo_median", s);
    median(h->srt, h->smooth, np, h->sm);
  }
  {
    StageTimer st("stripe_vo_unsort", s);
    vo_unsort<<<dim3(ceil_div(h->nproj, 128), ni, nz), 128, 0, s>>>(h->tt, np, ni, h->smooth,
                                                                    h->ids, nullptr);
    vo_transpose<<<tgrid, tblk, 0, s>>>(tomo, pstride, zstride, h->tt, np, ni, 0);
  }
  TCB_LAUNCH_CHECK();
  count_launch(15);
  return TCB_OK;
}

extern "C" int tcb_stripe_vo_destroy(tcb_stripe_vo *h) {
  if (!h) return TCB_OK;
  vo_release(h);
  delete h;
  return TCB_OK;
}
