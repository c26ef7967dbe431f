/*
 * tomocupy_b200 — C ABI of the B200-native tomographic reconstruction kernels.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as void*; NULL means the legacy default stream), enqueues its work
 * asynchronously on that stream, and returns a tcb_status.  On a non-zero
 * status tcb_last_error() returns a message for the calling thread.
 *
 * Operators mirror the reference's SWIG classes (src/cuda/*.i): an opaque
 * handle replaces the C++ object, *_create replaces the constructor,
 * *_destroy replaces free()/the destructor, and one function exists per
 * method.  A precision argument (TCB_FLOAT32 / TCB_FLOAT16) replaces the
 * reference's split into cfunc_X and cfunc_Xfp16 modules: FLOAT16 means fp16
 * storage of the caller's buffers with fp32 arithmetic inside the kernels.
 *
 * Handles are not re-entrant across concurrently running streams (they own
 * scratch memory), exactly like the reference objects.
 */
#ifndef TOMOCUPY_B200_H
#define TOMOCUPY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TCB_OK = 0,
  TCB_ERR_INVALID_ARGUMENT = 1,
  TCB_ERR_CUDA = 2,
  TCB_ERR_CUFFT = 3,
  TCB_ERR_OUT_OF_MEMORY = 4,
  TCB_ERR_NOT_SUPPORTED = 5,
  TCB_ERR_FREED = 6
} tcb_status;

typedef enum { TCB_FLOAT32 = 0, TCB_FLOAT16 = 1 } tcb_precision;

/* Element type of raw detector frames. */
typedef enum { TCB_U8 = 0, TCB_U16 = 1, TCB_F32 = 2 } tcb_dtype;

/* Message describing the last failure on this thread ("" if none). */
const char *tcb_last_error(void);
/* Library ABI version (major*100 + minor). */
int tcb_version(void);

/* Instrumentation (no counterpart in the reference, which has no profiling
 * hooks).  tcb_profile_enable(1) clears and starts recording a CUDA event
 * pair around every native stage launch (on the stream it is launched on);
 * tcb_profile_report synchronises the recorded events and writes JSON
 * {"stage": {"count": c, "ms": total, "bytes": b, "flops": f}, ...} into
 * buf, where b and f sum the algorithmic DRAM bytes and FLOPs that a stage
 * states for its launches (0 where it states none).  tcb_launch_count
 * returns the number of native kernel launches since process start (cuFFT
 * launches are not counted). */
int tcb_profile_enable(int on);
int tcb_profile_report(char *buf, size_t len);
int tcb_launch_count(uint64_t *out);

/* Failure-detection check (no counterpart in the reference, whose kernels
 * have no waits).  Runs the bounded mbarrier wait that the tensor-core and
 * TMA kernels use (tcb_tcfilter_status, tcb_fourierrec_status and
 * tcb_linerec_status report its expiry) on an mbarrier that nothing
 * arrives on, with a budget of budget_cycles SM clock cycles: *timed_out
 * is 1 when the wait gave up (always, by construction) and *waited_cycles
 * how long it waited.  Synchronous on the stream; the context stays usable. */
int tcb_check_bounded_wait(long long budget_cycles, int *timed_out, long long *waited_cycles,
                           void *stream);

/* Asynchronous 2D copy (host<->device or device<->device, direction inferred
 * from the pointers): height rows of width_bytes, with row pitches in bytes.
 * The chunk conveyor uses it to move [nproj, ncz, n] slabs of a
 * [nproj, nz, n] stack without a host-side repack; it replaces the pinned
 * staging copies of GPURec.recon_all (src/tomocupy/rec.py:184-195). */
int tcb_copy2d(void *dst, size_t dpitch, const void *src, size_t spitch,
               size_t width_bytes, size_t height, void *stream);

/* ------------------------------------------------------------------------
 * Pre-processing: dark/flat normalisation and -log.
 * ------------------------------------------------------------------------ */

/* Flat/dark reductions for one chunk of rows.
 * Replaces the mean part of ProcFunctions.darkflat_correction
 * (src/tomocupy/processing/proc_functions.py:55-74).
 *   dark  [ndark, nz, n], flat [nflat, nz, n] of type in_dtype
 *   dark0 [nz, n] fp32 = mean_k dark[k]
 *   flat_linear == 0: flat0 [nz, n] fp32 = mean_k(flat[k]/bright_ratio)*(1+1e-5) - dark0
 *   flat_linear != 0: flat0 = mean of flat[:nflat/2]/bright_ratio,
 *                     flat1 = mean of flat[nflat/2+1:]/bright_ratio (unscaled;
 *                     the per-angle blend happens in tcb_prep_rows). */
int tcb_darkflat_stats(void *dark0, void *flat0, void *flat1, const void *dark,
                       const void *flat, size_t ndark, size_t nflat, size_t nz,
                       size_t n, int in_dtype, float bright_ratio, int flat_linear,
                       void *stream);

/* Prep flags. */
#define TCB_PREP_DARKFLAT 1u   /* apply (x - dark0)/flat0                        */
#define TCB_PREP_MINUS_LOG 2u  /* where(x<=0,1,x) -> -log -> nan_to_num(6,0,0)   */
#define TCB_PREP_FLAT_LINEAR 4u /* flat0/flat1 are the two half-means            */
#define TCB_PREP_EDGE_PAD 8u   /* replicate first/last column into the padding   */

/* One fused pass over rows: reads input row (p, z) of a [nproj, nz, n]
 * frame stack (in_dtype; TCB_F32 when the input is already normalised) and
 * writes output row (z, p) in sinogram order:
 *   out[z*out_zstride + (p+out_poff)*out_pstride + out_xoff + x]
 * with the columns [0, out_xoff) and [out_xoff+n, out_width) filled with the
 * edge values when TCB_PREP_EDGE_PAD is set.  in_zstride/in_pstride describe
 * the input layout in elements.  Replaces darkflat_correction + minus_log +
 * the swapaxes copy (rec.py:174) + the edge padding of fbp_filter_center
 * (reconstruction/backproj_functions.py:93-109). */
int tcb_prep_rows(float *out, const void *in, const float *dark0, const float *flat0,
                  const float *flat1, size_t nproj, size_t nz, size_t n,
                  size_t in_pstride, size_t in_zstride, int in_dtype,
                  size_t out_zstride, size_t out_pstride, size_t out_poff,
                  size_t out_xoff, size_t out_width, unsigned flags, void *stream);

/* Dark/flat normalisation (+ optional -log and edge padding) of a contiguous
 * [nproj, nz, n] frame stack, exactly as tcb_darkflat_stats followed by
 * tcb_prep_rows (flat_linear excluded), but without any device allocation.
 * This entry point has no counterpart in the reference.  It is for callers
 * that cannot allocate device memory where they normalise frames (e.g. an
 * acquisition loop that must not allocate once streaming, or code inside a
 * runtime that owns the device allocator).  The dark/flat statistics live in
 * a fixed array inside the library (2 * TCB_NOALLOC_MAX_PLANE floats, 8 MiB
 * per device, kept until the process exits); nz*n above
 * TCB_NOALLOC_MAX_PLANE is rejected with TCB_ERR_INVALID_ARGUMENT.  All
 * calls share that array: calls that overlap on the GPU race.  The first call
 * on each device looks up the array's address with that device current; make
 * it before any stream capture.  Inputs and outputs are the caller's. */
#define TCB_NOALLOC_MAX_PLANE (1u << 20)
int tcb_prep_noalloc(float *out, const void *data, const void *dark, const void *flat,
                     size_t nproj, size_t nz, size_t n, size_t ndark, size_t nflat,
                     int in_dtype, float bright_ratio, size_t out_zstride,
                     size_t out_pstride, size_t out_poff, size_t out_xoff,
                     size_t out_width, unsigned flags, void *stream);

/* Binning.  Replaces utils.downsample (src/tomocupy/utils.py:157-167) as the
 * reader applies it to chunks of projections, darks and flats
 * (src/tomocupy/dataio/reader.py:335-356): out float32 [nframes, nz, n] =
 * sums of 2^binning x 2^binning blocks of in (frames of nz * 2^binning rows of
 * n * 2^binning samples, frame and row strides in elements), columns then
 * rows as pairwise float32 trees, the reference's order.  binning in [1, 4]. */
int tcb_downsample(float *out, const void *in, int in_dtype, size_t nframes, size_t nz, size_t n,
                   size_t in_fstride, size_t in_zstride, int binning, void *stream);

/* Double-field-of-view padding.  Replaces ProcFunctions.pad360
 * (src/tomocupy/processing/proc_functions.py:109-124), applied by proc_proj
 * after -log when file_type is 'double_fov' (proc_functions.py:190-193).
 * weights: the smooth transition v of length w into v (host, float64).
 * rows: in place on nrows rows whose first ni floats hold the samples (row
 * stride row_stride >= 2 ni): optional flip, the last w samples times v
 * (device, float64), zeros in [ni, 2 ni). */
int tcb_pad360_weights(double *v, size_t w);
int tcb_pad360_rows(float *rows, size_t nrows, size_t ni, size_t row_stride, int flip,
                    const double *v, size_t w, void *stream);

/* Projection rotation.  Replaces ProcFunctions.rotate_proj
 * (src/tomocupy/processing/proc_functions.py:126-138), applied by proc_proj
 * after phase retrieval and before -log when rotate_proj_angle != 0
 * (proc_functions.py:181-183): ndimage.rotate(data, angle, reshape=False,
 * order, axes=(2, 1), mode='nearest').  out[f] (frame stride out_fstride)
 * gets in[f] (frame stride in_fstride; nz rows of n floats) sampled at
 * iz = offz + oz c + ox s, ix = offx - oz s + ox c, clamped to the plane,
 * with spline order 0 or 1, in float64 rounded to float32.  c, s: cosine
 * and sine of the angle; offz, offx: the offset that keeps the plane centre
 * fixed (both computed by the caller).  out and in must not overlap. */
int tcb_rotate_proj(float *out, const float *in, size_t nframes, size_t nz, size_t n,
                    size_t in_fstride, size_t out_fstride, double c, double s, double offz,
                    double offx, int order, void *stream);

/* Outlier (zinger) removal.  Replaces ProcFunctions.remove_outliers
 * (src/tomocupy/processing/proc_functions.py:96-107), which proc_sino applies
 * to the projections, darks and flats of a chunk before dark/flat correction
 * (proc_functions.py:146-148): out = where(in > f and in - f > threshold, f,
 * in) with f = median_filter(in, [width, 1, width]) (mode 'reflect') over
 * frames [nframes, nz, n] of type in_dtype (frame and row strides of the
 * input in elements; out is contiguous with in's type).  Out of place.
 * width in [1, 11]. */
int tcb_dezinger(void *out, const void *in, int in_dtype, size_t nframes, size_t nz, size_t n,
                 size_t in_fstride, size_t in_zstride, int width, double threshold,
                 void *stream);

/* ------------------------------------------------------------------------
 * Fourier-wavelet ring removal.  Replaces remove_stripe_fw with DWTForward /
 * DWTInverse / afb1d / sfb1d (src/tomocupy/processing/remove_stripe.py:51-293).
 * create: sizes of the sinogram chunk, DWT levels, damping sigma and the
 * wavelet filter bank (host float64 arrays of length L, PyWavelets order).
 * apply_sino: in place on padded sinograms [nz][nproj + nproj/8][ni] (slice
 * stride sstride), data rows starting at (nproj/8)/2, other rows zero.
 * ------------------------------------------------------------------------ */
typedef struct tcb_stripe_fw tcb_stripe_fw;
int tcb_stripe_fw_create(tcb_stripe_fw **out, size_t nproj, size_t nz, size_t ni, int level,
                         float sigma, const double *dec_lo, const double *dec_hi,
                         const double *rec_lo, const double *rec_hi, int L);
int tcb_stripe_fw_apply_sino(tcb_stripe_fw *h, float *sino, size_t sstride, void *stream);
int tcb_stripe_fw_destroy(tcb_stripe_fw *h);

/* Titarenko ring removal.  Replaces remove_stripe_ti
 * (src/tomocupy/processing/remove_stripe.py:296-307), called by
 * ProcFunctions.proc_sino for remove_stripe_method 'ti'
 * (src/tomocupy/processing/proc_functions.py:154-156).  mask: the column
 * range [m0, m1) that the reference's mask[:, n//2 - ms//2 : n//2 + ms//2]
 * selects (ms = mask_size * n, Python slice rules; host only; the reference
 * slices with a float when mask_size is a float, which NumPy and CuPy
 * reject, so only integer mask sizes run there).  n must be even (for odd n
 * the reference's irfft returns n - 1 samples and its add fails).
 * apply_sino: in place on
 * sino[z * zstride + p * pstride + x] (nz slices, nproj angles, n columns).
 * ------------------------------------------------------------------------ */
typedef struct tcb_stripe_ti tcb_stripe_ti;
int tcb_stripe_ti_mask(size_t n, double mask_size, long long *m0, long long *m1);
int tcb_stripe_ti_create(tcb_stripe_ti **out, size_t nproj, size_t nz, size_t n, double beta,
                         double mask_size);
int tcb_stripe_ti_apply_sino(tcb_stripe_ti *h, float *sino, size_t zstride, size_t pstride,
                             void *stream);
int tcb_stripe_ti_destroy(tcb_stripe_ti *h);

/* Vo's all-stripe ring removal.  Replaces remove_all_stripe with _rs_dead3,
 * _rs_large3, _rs_sort3 and _detect_stripe_batch
 * (src/tomocupy/processing/remove_stripe.py:311-498), called by
 * ProcFunctions.proc_sino for remove_stripe_method 'vo-all'
 * (src/tomocupy/processing/proc_functions.py:157-159) with vo_all_snr,
 * vo_all_la_size, vo_all_sm_size and vo_all_dim.  create: chunk shape
 * (nproj in [12, 8192], ni in [8, 8192]), odd median windows <= 127, dim 1
 * (windows along the detector; dim 2 is not supported).  apply: in place on
 * tomo[p * pstride + z * zstride + x] (nproj angles, nz rows, ni columns).
 * Sorts along the angles are stable, as CuPy's argsort. */
typedef struct tcb_stripe_vo tcb_stripe_vo;
int tcb_stripe_vo_create(tcb_stripe_vo **out, size_t nproj, size_t nz, size_t ni, double snr,
                         int la_size, int sm_size, int dim);
int tcb_stripe_vo_apply(tcb_stripe_vo *h, float *tomo, size_t pstride, size_t zstride,
                        void *stream);
int tcb_stripe_vo_destroy(tcb_stripe_vo *h);

/* ------------------------------------------------------------------------
 * Single-distance phase retrieval of projections.  Replaces paganin_filter
 * (methods 'paganin', 'Gpaganin') and farago_filter
 * (src/tomocupy/processing/retrieve_phase.py:57-145), called by
 * ProcFunctions.proc_proj (src/tomocupy/processing/proc_functions.py:169-181).
 * Units as in those functions: pixel_size and dist in cm, energy in keV,
 * W in cm.  pads: the edge padding (rows py, columns pz, each side) that
 * _calc_pad chooses (retrieve_phase.py:178-206); host only.
 * create: batch = projections per transform batch; the filter is built on
 * the host.  apply: in place on nproj projections [nproj, dy, dz] float32
 * (the reference's data[m] = proj).  Not re-entrant across streams (the
 * handle owns the padded batch and its spectra).
 * ------------------------------------------------------------------------ */
#define TCB_PHASE_PAGANIN 0
#define TCB_PHASE_GPAGANIN 1
#define TCB_PHASE_FARAGO 2
typedef struct tcb_phase tcb_phase;
int tcb_phase_pads(size_t dy, size_t dz, double pixel_size, double dist, double energy,
                   int pad, size_t *py, size_t *pz);
int tcb_phase_create(tcb_phase **out, size_t batch, size_t dy, size_t dz, int method,
                     double pixel_size, double dist, double energy, double alpha, double db,
                     double W, int pad);
int tcb_phase_sizes(tcb_phase *h, size_t *py, size_t *pz);
int tcb_phase_apply(tcb_phase *h, float *data, size_t nproj, void *stream);
int tcb_phase_destroy(tcb_phase *h);

/* ------------------------------------------------------------------------
 * FBP filter.  Replaces cfunc_filter (src/include/cfunc_filter.cuh:9-23,
 * src/cuda/cfunc_filter.i:9-21): g real [nz, nproj, n] filtered in place
 * with w complex [nz, n/2+1] (one spectrum per slice).
 * ------------------------------------------------------------------------ */
typedef struct tcb_filter tcb_filter;
int tcb_filter_create(tcb_filter **out, size_t nproj, size_t nz, size_t n,
                      int precision);
int tcb_filter_apply(tcb_filter *h, void *g, const void *w, void *stream);
int tcb_filter_destroy(tcb_filter *h);

/* ------------------------------------------------------------------------
 * Mixed-precision filter on the tensor cores.  Same operator as
 * fbp_filter_center (src/tomocupy/reconstruction/backproj_functions.py:93-109:
 * edge pad to ne, R2C, x w, C2R, crop) followed by cfunc_filter::filter
 * (src/cuda/cfunc_filter.cu:49-61), written as the n x n matrix it is and
 * applied as an fp16 tcgen05 GEMM with fp32 accumulation and a hi/lo
 * split-precision correction (x_hi T_hi + x_lo T_hi + x_hi T_lo).  The
 * reference's own half-precision path is cfunc_filterfp16 (fp16 cuFFT).
 *
 * create: nproj angles, up to nz slices per apply call, n columns
 *   (n >= 64, n % 8 == 0), nkern distinct filter kernels (1 = shared by all
 *   slices; otherwise slice z of a call uses kernel kern0 + z).
 * set_kernels: hz host float64 [nkern][ne], the unnormalised C2R of each
 *   kernel's spectrum w (ne = padded length, pad = left padding = ne/2 - n/2
 *   in the reference); synchronous.
 * tcb_prep_rows_split16 (below) writes the hi/lo operand planes.
 * apply: x_hi/x_lo fp16 [nz * nproj][lda] (z-major rows).  out_mode
 *   TCB_TCF_OUT_ROWS writes fp32 out[(z*nproj + p)*ldo + j];
 *   TCB_TCF_OUT_PAIRS writes the packed complex layout of
 *   FourierRec.backprojection (src/tomocupy/reconstruction/fourierrec.py:63-68):
 *   float2 out[(z % (nz/2))*nproj + p][j], real part from slices < nz/2.
 * status: 1 in *timed_out when a kernel gave up on a bounded wait (synchronous).
 * ------------------------------------------------------------------------ */
typedef struct tcb_tcfilter tcb_tcfilter;
#define TCB_TCF_OUT_ROWS 0
#define TCB_TCF_OUT_PAIRS 1
int tcb_tcfilter_create(tcb_tcfilter **out, size_t nproj, size_t nz, size_t n, size_t nkern);
int tcb_tcfilter_set_kernels(tcb_tcfilter *h, const double *hz, size_t ne, size_t pad,
                             void *stream);
int tcb_tcfilter_apply(tcb_tcfilter *h, const void *x_hi, const void *x_lo, size_t lda,
                       size_t nz, size_t kern0, void *out, int out_mode, size_t ldo,
                       void *stream);
int tcb_tcfilter_status(tcb_tcfilter *h, int *timed_out);
int tcb_tcfilter_destroy(tcb_tcfilter *h);

/* ------------------------------------------------------------------------
 * Fused fp32 filter.  Same operator as fbp_filter_center
 * (src/tomocupy/reconstruction/backproj_functions.py:93-109: edge pad to ne,
 * R2C, x w, C2R, crop) with cfunc_filter::filter
 * (src/cuda/cfunc_filter.cu:49-61), computed as a circular convolution of
 * length L = the power of two >= 2n (two FFTs in shared memory) plus the
 * folded edge-padding columns, for two slices per complex transform.
 *
 * create: nproj angles, up to nz slices per apply call, n columns
 *   (2 <= n <= 4096), nkern filter kernels (1 = shared; otherwise slice z of
 *   a call uses kernel kern0 + z).
 * set_kernels: hz host float64 [nkern][ne], the unnormalised C2R of each
 *   kernel's spectrum w, pad = left padding (ne/2 - n/2 in the reference);
 *   synchronous.  Same arguments as tcb_tcfilter_set_kernels.
 * apply: x fp32 rows x[(z*nproj + p)*ldx + xoff + i], i < n (not modified).
 *   Slices z < half = ceil(nz/2) pair with slice z + half.
 *   TCB_FFF_OUT_ROWS: fp32 out[(z*nproj + p)*ldo + j].
 *   TCB_FFF_OUT_PAIRS (nz even): float2 out[(z*nproj + p)*n + j], z < nz/2,
 *     the packed layout of FourierRec.backprojection
 *     (src/tomocupy/reconstruction/fourierrec.py:63-68).
 *   TCB_FFF_OUT_SPECTRUM (nz even, n a power of two >= 256): the forward
 *     length-n DFT of each packed row, i.e. the projection FFT of
 *     cfunc_fourierrec::backprojection (src/cuda/cfunc_fourierrec.cu:67-94);
 *     pass it to a fourierrec handle with tcb_fourierrec_set_input_spectrum.
 * ------------------------------------------------------------------------ */
typedef struct tcb_fftfilter tcb_fftfilter;
#define TCB_FFF_OUT_ROWS 0
#define TCB_FFF_OUT_PAIRS 1
#define TCB_FFF_OUT_SPECTRUM 2
int tcb_fftfilter_create(tcb_fftfilter **out, size_t nproj, size_t nz, size_t n, size_t nkern);
int tcb_fftfilter_set_kernels(tcb_fftfilter *h, const double *hz, size_t ne, size_t pad,
                              void *stream);
int tcb_fftfilter_apply(tcb_fftfilter *h, const float *x, size_t ldx, size_t xoff, size_t nz,
                        size_t kern0, void *out, int out_mode, size_t ldo, void *stream);
int tcb_fftfilter_destroy(tcb_fftfilter *h);

/* Split-fp16 variant of tcb_prep_rows (same normalisation chain, same
 * reference lines), written as hi = fp16(v) and lo = fp16(v - hi) planes
 * [z*out_zstride + p*out_pstride + x]; no edge padding (the tensor-core
 * filter folds it into its operator). */
int tcb_prep_rows_split16(void *hi, void *lo, const void *in, const float *dark0,
                          const float *flat0, const float *flat1, size_t nproj, size_t nz,
                          size_t n, size_t in_pstride, size_t in_zstride, int in_dtype,
                          size_t out_zstride, size_t out_pstride, unsigned flags,
                          void *stream);

/* ------------------------------------------------------------------------
 * Fourier-gridding backprojector.  Replaces cfunc_fourierrec
 * (src/include/cfunc_fourierrec.cuh:10-36, src/cuda/cfunc_fourierrec.i:9-21).
 *   theta: device fp32 [nproj] (read during create only, as in the reference)
 *   nz:    number of complex slice pairs
 * ------------------------------------------------------------------------ */
typedef struct tcb_fourierrec tcb_fourierrec;
int tcb_fourierrec_create(tcb_fourierrec **out, size_t nproj, size_t nz, size_t n,
                          const float *theta, int precision);
/* cfunc_fourierrec::backprojection: g complex [nz, nproj, n] (overwritten,
 * as in the reference), f complex [nz, n, n]. */
int tcb_fourierrec_backprojection(tcb_fourierrec *h, void *f, void *g, void *stream);
/* Same reconstruction with the real/imaginary unpacking of
 * FourierRec.backprojection (reconstruction/fourierrec.py:61-68) fused in:
 * f real [2*nz, n, n] (slice k = real part of pair k, slice nz+k = imaginary). */
int tcb_fourierrec_backprojection_slices(tcb_fourierrec *h, void *f, void *g,
                                         void *stream);
/* Pack 2*nz filtered real sinograms into nz complex pairs, cropping columns
 * [xoff, xoff+n) from rows of length row_stride:
 *   g[k, p, x] = src[k, p, xoff+x] + i*src[k+nz, p, xoff+x]
 * (reconstruction/fourierrec.py:63-64 plus the crop of
 * backproj_functions.py:107). */
int tcb_fourierrec_pack(tcb_fourierrec *h, void *g, const void *src,
                        size_t row_stride, size_t xoff, void *stream);
/* Tuning knob (no reference counterpart): slice pairs accumulated per
 * gridding block, 2/4/8/16, or 0 for the largest that the handle's nz allows.
 * Results do not depend on it beyond fp32 summation order. */
int tcb_fourierrec_set_pairs_per_block(tcb_fourierrec *h, int pairs);
/* Gridding mode (no reference counterpart).  TCB_GRID_FP32: the fp32
 * register-accumulation gridding (default; the drop-in).  TCB_GRID_TENSOR:
 * mixed precision on the tensor cores -- footprint weights and the spectrum
 * values (power-of-two scaled) in fp16, fp32 accumulation in TMEM, 32 slice
 * pairs per weight matrix; used by the mixed-precision path.
 * TCB_GRID_TENSOR_FP32: the fp32 drop-in on the tensor cores -- the weights of
 * 16 x 16-cell tiles and chunks of 64 samples precomputed once (split fp16
 * hi/lo images, about 64 KB per chunk: 9 GB at 2048 x 1500) and streamed by
 * bulk copies, the spectrum split into fp16 hi/lo rows per call and
 * gathered by cp.async, W_hi V_hi + W_lo V_hi + W_hi V_lo accumulated in fp32
 * in TMEM (within 1e-5 of the reference).  TCB_GRID_TENSOR_STREAM: the same
 * with fp16 weights and values only (mixed precision, half the tables).
 * Both return TCB_ERR_OUT_OF_MEMORY when the tables do not fit (the handle
 * keeps its previous mode).  status: 1 in *timed_out when a tensor-core
 * gridding wait gave up (synchronous). */
#define TCB_GRID_FP32 0
#define TCB_GRID_TENSOR 1
#define TCB_GRID_TENSOR_FP32 2
#define TCB_GRID_TENSOR_STREAM 3
int tcb_fourierrec_set_gridding(tcb_fourierrec *h, int mode);
/* Output precision (no reference counterpart): TCB_FLOAT16 writes the
 * reconstructed slices in fp16 while the input g stays fp32 (a FLOAT16 handle
 * has fp16 input and output). */
int tcb_fourierrec_set_output(tcb_fourierrec *h, int precision);
/* Input form (no reference counterpart): on != 0 means g already holds the
 * forward length-n DFT of every packed projection row (what
 * tcb_fftfilter_apply writes with TCB_FFF_OUT_SPECTRUM), so the projection
 * FFT is skipped.  FLOAT32 handles only. */
int tcb_fourierrec_set_input_spectrum(tcb_fourierrec *h, int on);
int tcb_fourierrec_status(tcb_fourierrec *h, int *timed_out);
/* Sample positions (test hook for bit-exact indexing): x, y fp32 [nproj, n]
 * are the polar sample coordinates that takexy computes
 * (src/include/kernels_fourierrec.cuh:23-36, same layout), fx, fy int32
 * [nproj, n] the floor(2n x), floor(2n y) that place each sample's 9 x 9
 * footprint (kernels_fourierrec.cuh:84-85 adds -m), all as the gridding
 * kernels of this handle compute them. */
int tcb_fourierrec_sample_positions(tcb_fourierrec *h, float *x, float *y, int *fx, int *fy,
                                    void *stream);
int tcb_fourierrec_destroy(tcb_fourierrec *h);

/* ------------------------------------------------------------------------
 * Line backprojector.  Replaces cfunc_linerec
 * (src/include/cfunc_linerec.cuh:9-23, src/cuda/cfunc_linerec.i:9-25).
 * All methods accumulate into f [ncz, n, n]; g is [nz, ncproj, n].
 * ------------------------------------------------------------------------ */
typedef struct tcb_linerec tcb_linerec;
int tcb_linerec_create(tcb_linerec **out, size_t nproj, size_t nz, size_t n,
                       size_t ncproj, size_t ncz, int precision);
int tcb_linerec_backprojection(tcb_linerec *h, void *f, const void *g,
                               const float *theta, float phi, int sz, void *stream);
int tcb_linerec_backprojection_try(tcb_linerec *h, void *f, const void *g,
                                   const float *theta, const float *sh, float phi,
                                   int sz, void *stream);
int tcb_linerec_backprojection_try_lamino(tcb_linerec *h, void *f, const void *g,
                                          const float *theta, const float *phi,
                                          int sz, void *stream);
/* status (no reference counterpart): 1 in *timed_out when a TMA wait of the
 * float32 backprojection gave up (synchronous). */
int tcb_linerec_status(tcb_linerec *h, int *timed_out);
int tcb_linerec_destroy(tcb_linerec *h);

/* ------------------------------------------------------------------------
 * Log-polar backprojector.  Replaces cfunc_lprec
 * (src/include/cfunc_lprec.cuh:9-49, src/cuda/cfunc_lprec.i:11-29).
 * setgrids borrows the caller's device grids for the handle's lifetime (as
 * the reference does); backprojection zeroes f [nz, n, n] and accumulates
 * the three spans; g [nz, nproj, n] is overwritten by its spline
 * coefficients (as in the reference).
 * ------------------------------------------------------------------------ */
typedef struct tcb_lprec tcb_lprec;
int tcb_lprec_create(tcb_lprec **out, size_t nproj, size_t nz, size_t n, size_t ntheta,
                     size_t nrho, int precision);
int tcb_lprec_setgrids(tcb_lprec *h, const void *fz, const float *lp2p1, const float *lp2p2,
                       const float *lp2p1w, const float *lp2p2w, const float *C2lp1,
                       const float *C2lp2, const int *lpids, const int *wids,
                       const int *cids, size_t nlpids, size_t nwids, size_t ncids);
int tcb_lprec_backprojection(tcb_lprec *h, void *f, void *g, void *stream);
int tcb_lprec_destroy(tcb_lprec *h);

/* ------------------------------------------------------------------------
 * Laminography Fourier chain.
 * ------------------------------------------------------------------------ */

/* Replaces cfunc_fft2d (src/include/cfunc_fft2d.cuh:7-26, src/cuda/cfunc_fft2d.i:9-18).
 * fwd: g complex [ntheta, deth, detw/2+1] <- f real [ntheta, deth, detw]
 * (f is sign-flipped in place, as in the reference). */
typedef struct tcb_fft2d tcb_fft2d;
int tcb_fft2d_create(tcb_fft2d **out, size_t ntheta, size_t detw, size_t deth);
int tcb_fft2d_fwd(tcb_fft2d *h, void *g, void *f, void *stream);
int tcb_fft2d_destroy(tcb_fft2d *h);

/* Replaces cfunc_usfft2d (src/include/cfunc_usfft2d.cuh:7-33,
 * src/cuda/cfunc_usfft2d.i:9-18); constructor arguments in the reference's
 * Python order (n0, n1, n2) = (slabs per call, grid y, grid x).
 * adj: f complex [n1][n0][n2] (y, slab, x in the Python argument names)
 *      <- g complex [2*ntheta, deth, detw/2+1]
 * (the packed chunk of BackprojLamFourierParallel.usfft2d_chunks), theta
 * device fp32 [ntheta], chunk index k, full detector height deth0. */
typedef struct tcb_usfft2d tcb_usfft2d;
int tcb_usfft2d_create(tcb_usfft2d **out, size_t n0, size_t n1, size_t n2, size_t ntheta,
                       size_t detw, size_t deth);
int tcb_usfft2d_adj(tcb_usfft2d *h, void *f, const void *g, const float *theta, float phi,
                    int k, int deth0, void *stream);
/* Fused form: rows [row0, row0+nrows) of the whole stage-1 spectrum
 * S1 [ntheta, deth_full, detw/2+1] (conjugate mirror read in place) into
 * S2 [n1, deth_full/2+1, n0] at frequency rows row0.. (replaces the packing
 * of backproj_lamfourier_parallel.py:197-215 and the host copies). */
int tcb_usfft2d_adj_rows(tcb_usfft2d *h, void *S2, const void *S1, const float *theta,
                         float phi, int row0, int nrows, int deth_full, void *stream);
/* cfunc_usfft2d::fwd (src/cuda/cfunc_usfft2d.cu:53-70): g complex
 * [2*ntheta, deth, detw/2+1] in adj's packed layout (detector frequencies
 * above detw/2 mirrored into angle planes ntheta..) <- f complex [n1][n0][n2]
 * (the layout adj writes), chunk index k, full detector height deth0.
 * The adjoint of tcb_usfft2d_adj. */
int tcb_usfft2d_fwd(tcb_usfft2d *h, void *g, const void *f, const float *theta, float phi,
                    int k, int deth0, void *stream);
/* fp16 storage (no reference counterpart; the reference's laminography path
 * is fp32 only): TCB_FLOAT16 makes the stage-1 spectrum input and the output
 * of adj/adj_rows complex fp16 (__half2) arrays; gridding, FFTs and
 * deapodization compute in fp32.  in_scale (device, [ntheta], or NULL): the
 * input of angle t was stored multiplied by 1/in_scale[t] and is multiplied
 * back on load.  out_inv_scale (device, [rows of the output], or NULL): each
 * call multiplies its output by a power of two that keeps it below 2^14 and
 * writes the inverse factor for each of its rows there.  The arrays are the
 * caller's and must outlive the calls. */
int tcb_usfft2d_set_storage(tcb_usfft2d *h, int precision, const float *in_scale,
                            float *out_inv_scale);
/* Sample positions (test hook for bit-exact indexing): x, y fp32
 * [ntheta, deth, detw] as take_x computes them for chunk k and full height
 * deth0 (src/include/kernels_usfft2d.cu:5-18, same layout), with the
 * arithmetic of this handle's gridding kernel. */
int tcb_usfft2d_sample_positions(tcb_usfft2d *h, float *x, float *y, const float *theta,
                                 float phi, int k, int deth0, void *stream);
int tcb_usfft2d_destroy(tcb_usfft2d *h);

/* Replaces cfunc_usfft1d (src/include/cfunc_usfft1d.cuh:7-34,
 * src/cuda/cfunc_usfft1d.i:9-18); constructor in the reference's Python
 * order (n0, n1, n2, deth) = (height, rows per call, width, detector height).
 * adj: f real [n1, n0(height), n2(width)] <- g complex [n1, deth/2+1, n2]. */
typedef struct tcb_usfft1d tcb_usfft1d;
int tcb_usfft1d_create(tcb_usfft1d **out, size_t n0, size_t n1, size_t n2, size_t deth);
int tcb_usfft1d_adj(tcb_usfft1d *h, void *f, const void *g, float phi, void *stream);
/* cfunc_usfft1d::fwd (src/cuda/cfunc_usfft1d.cu:50-66): g complex
 * [n1, deth/2+1, n2] <- f real [n1, n0(height), n2(width)].  Row t of g is
 * computed from its own height z(t) for t <= deth/2 (the reference's kernel
 * also runs rows t > deth/2, which race to overwrite row deth - t with an
 * unconjugated value). */
int tcb_usfft1d_fwd(tcb_usfft1d *h, void *g, const void *f, float phi, void *stream);
/* fp16 storage of the input g (complex fp16); output and arithmetic fp32.
 * in_scale (device, [deth/2+1], or NULL): row r of g is multiplied by
 * in_scale[r] on load (the out_inv_scale rows written by usfft2d). */
int tcb_usfft1d_set_storage(tcb_usfft1d *h, int precision, const float *in_scale);
int tcb_usfft1d_destroy(tcb_usfft1d *h);

#ifdef __cplusplus
}
#endif
#endif /* TOMOCUPY_B200_H */
