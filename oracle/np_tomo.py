"""NumPy restatement of the reference reconstruction path (test oracle / CPU baseline).

Every function cites the reference code it restates.  ``dtype`` selects the
working precision: float32 reproduces the reference's arithmetic (with
NumPy's cos/sin/exp standing in for CUDA intrinsics), float64 is the
"accurate" oracle with the same algorithm and constants.  FFTs use
scipy.fft (multi-threaded via ``workers``); cuFFT's unnormalised inverse is
matched with ``norm="forward"``.
"""
from __future__ import annotations

import math
import os

import numpy as np
import scipy.fft as sfft

WORKERS = os.cpu_count() or 1


# --------------------------------------------------------------------------
# pre-processing (src/tomocupy/processing/proc_functions.py:55-83)
# --------------------------------------------------------------------------
def darkflat(data, dark, flat, bright_ratio=1.0):
    """(data - mean(dark)) / (mean(flat/bright_ratio)*f32(1+1e-5) - mean(dark)), float32."""
    dark0 = dark.astype(np.float32)
    flat0 = flat.astype(np.float32)
    flat0 = flat0 / np.float32(bright_ratio)
    flat0 = np.mean(flat0, axis=0, dtype=np.float32)
    dark0 = np.mean(dark0, axis=0, dtype=np.float32)
    flat0 = flat0 * np.float32(1 + 1e-5)
    flat0 = flat0 - dark0
    return (data.astype(np.float32) - dark0) / flat0


def darkflat_linear(data, dark, flat, bright_ratio=1.0):
    """flat_linear variant (proc_functions.py:62-66): float64 blend across angles."""
    nproj = data.shape[0]
    flat0 = flat.astype(np.float32) / np.float32(bright_ratio)
    p0 = np.mean(flat0[:flat0.shape[0] // 2], axis=0, dtype=np.float32)
    p1 = np.mean(flat0[flat0.shape[0] // 2 + 1:], axis=0, dtype=np.float32)
    v = np.linspace(0, 1, nproj)[..., np.newaxis, np.newaxis]
    f = (1 - v) * p0 + v * p1
    dark0 = np.mean(dark.astype(np.float32), axis=0, dtype=np.float32)
    f = f * np.float64(np.float32(1 + 1e-5))
    f = f - dark0
    return ((data.astype(np.float32) - dark0) / f).astype(np.float32)


def dezinger(data, width, threshold):
    """ProcFunctions.remove_outliers (proc_functions.py:96-107): median over
    [width, 1, width] (scipy.ndimage.median_filter, mode 'reflect', the same
    rank filter as cupyx's), pixels more than threshold above it replaced.
    Returns a new array of data's type."""
    import scipy.ndimage as ndi
    data = np.array(data)
    f = ndi.median_filter(data, [width, 1, width])
    return np.where(np.logical_and(data > f, (data - f) > threshold), f, data)


def downsample(data, binning):
    """utils.downsample (utils.py:157-167) on float32 frames: b times the sum of
    even and odd columns, then b times the sum of even and odd rows."""
    data = np.asarray(data, dtype=np.float32)
    for _ in range(binning):
        data = data[:, :, ::2] + data[:, :, 1::2]
    for _ in range(binning):
        data = data[:, ::2] + data[:, 1::2]
    return data


def pad360(data, centeri, ni, center):
    """ProcFunctions.pad360 (proc_functions.py:109-124) on float32
    [nproj, nz, ni]: flip when centeri < ni // 2, the last w = max(1,
    int(2 (ni - center))) columns times the float64 transition
    v**5 (126 - 420 v + 540 v**2 - 315 v**3 + 70 v**4), v = linspace(1, 0, w,
    endpoint=False), then zeros up to 2 ni columns.  Returns a new array."""
    data = np.array(data, dtype=np.float32)
    if centeri < ni // 2:
        data[:] = data[:, :, ::-1]
    w = max(1, int(2 * (ni - center)))
    v = np.linspace(1, 0, w, endpoint=False)
    v = v ** 5 * (126 - 420 * v + 540 * v ** 2 - 315 * v ** 3 + 70 * v ** 4)
    data[:, :, -w:] *= v
    return np.pad(data, ((0, 0), (0, 0), (0, data.shape[-1])), "constant")


def minus_log(x):
    """where(x<=0 -> 1), -log, nan_to_num(nan=6, posinf=0, neginf=0)."""
    x = np.where(x <= 0, np.float32(1.0), x).astype(np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = -np.log(x)
    return np.nan_to_num(r, nan=6.0, posinf=0.0, neginf=0.0).astype(np.float32)


# --------------------------------------------------------------------------
# Titarenko ring removal (src/tomocupy/processing/remove_stripe.py:296-307)
# --------------------------------------------------------------------------
class NumpyFFT:
    """The real FFTs the restatements call, as NumPy computes them (float32
    in -> complex64 out, complex64 in -> float32 out, float64 as float64).
    The reference calls cupy.fft, i.e. cuFFT, with the same types; a caller
    may pass another provider with these two methods (e.g. cuFFT through
    torch) to reproduce the reference's transforms more closely."""

    @staticmethod
    def rfft(a, axis=-1):
        return np.fft.rfft(a, axis=axis)

    @staticmethod
    def irfft(a, n, axis=-1):
        return np.fft.irfft(a, n, axis=axis)


def remove_stripe_ti(data, beta, mask_size, fft=NumpyFFT):
    """remove_stripe_ti on float32 [nproj, nz, n] (returns a new array): float32
    column means over angles minus column 0, convolution with
    gamma = beta * ((1-beta)/(1+beta))**|k| (gamma[0] -= 1) through
    rfft / irfft (complex64 times complex128, as CuPy types them), added to
    every angle inside mask[:, n//2 - ms//2 : n//2 + ms//2], ms = mask_size*n."""
    data = np.array(data, dtype=np.float32)
    n = data.shape[-1]
    gamma = beta * ((1 - beta) / (1 + beta)) ** np.abs(np.fft.fftfreq(n) * n)
    gamma[0] -= 1
    v = np.mean(data, axis=0, dtype=np.float32)
    v = v - v[:, 0:1]
    v = fft.irfft(fft.rfft(v).astype(np.complex64) * fft.rfft(gamma), n)
    mask = np.zeros(v.shape, dtype=v.dtype)
    ms = mask_size * mask.shape[1]
    mask[:, mask.shape[1] // 2 - int(ms // 2):mask.shape[1] // 2 + int(ms // 2)] = 1
    data[:] += v * mask
    return data


# --------------------------------------------------------------------------
# Vo's all-stripe removal (src/tomocupy/processing/remove_stripe.py:311-498)
# --------------------------------------------------------------------------
def _vo_detect(listfact, snr):
    """_detect_stripe_batch (remove_stripe.py:346-370) on [nz, ni] float32: per
    row, a least-squares line through the middle of the descending sort
    (dropping a quarter at each end), a noise level from its ends, and the
    columns beyond snr/2 noise levels above the line's start or below its
    end (only when the row's extreme passes snr)."""
    nz, num = listfact.shape
    srt = np.sort(listfact, axis=1)[:, ::-1]
    xl = np.arange(num, dtype=np.float32)
    nd = int(0.25 * num)
    x = xl[nd:-nd - 1]
    y = srt[:, nd:-nd - 1]
    n = x.size
    xm = float(x.mean())
    ym = y.mean(axis=1)
    sxy = (y * x).sum(axis=1) - n * ym * xm
    sxx = float((x ** 2).sum() - n * xm ** 2)
    slope = sxy / sxx
    icpt = ym - slope * xm
    numt1 = icpt + slope * xl[-1]
    noise = np.clip(np.abs(numt1 - icpt), 1e-6, None)
    val1 = np.abs(srt[:, 0] - icpt) / noise
    val2 = np.abs(srt[:, -1] - numt1) / noise
    mask = np.zeros((nz, num), dtype=np.float32)
    upper = (icpt + noise * snr * 0.5)[:, None]
    lower = (numt1 - noise * snr * 0.5)[:, None]
    mask = np.where((val1 >= snr)[:, None] & (listfact > upper), 1.0, mask)
    mask = np.where((val2 >= snr)[:, None] & (listfact <= lower), 1.0, mask)
    return mask


def _vo_dilate(mask):
    """binary_dilation with a (1, 3) structure, one iteration: a column is set
    when it or a neighbour along the detector is set."""
    import scipy.ndimage as ndi
    return ndi.binary_dilation(mask, iterations=1,
                               structure=np.ones((1, 3), dtype=bool)).astype(mask.dtype)


def _vo_sort_t(tomo):
    """The reference's sort along the angles: on the [ni, nz, nproj] transpose,
    a stable argsort and the sorted values (C-contiguous in that order)."""
    t = np.transpose(tomo, (2, 1, 0))
    ids = np.argsort(t, axis=2, kind="stable")
    return np.take_along_axis(t, ids, axis=2), ids


def _vo_unsort_t(vals_t, ids):
    """Inverse of _vo_sort_t on [ni, nz, nproj] values, back to [nproj, nz, ni]."""
    inv = np.empty_like(ids)
    np.put_along_axis(inv, ids, np.broadcast_to(np.arange(ids.shape[2], dtype=ids.dtype),
                                                ids.shape), axis=2)
    return np.transpose(np.take_along_axis(vals_t, inv, axis=2), (2, 1, 0))


def _vo_large(tomo, snr, size, drop_ratio=0.1):
    """_rs_large3 (remove_stripe.py:388-424) on [nproj, nz, ni], with the
    reference's array layouts (the float32 means reduce in the same order)."""
    import scipy.ndimage as ndi
    drop_ratio = max(min(drop_ratio, 0.8), 0)
    nproj = tomo.shape[0]
    ndrop = int(0.5 * drop_ratio * nproj)
    srt_t, ids = _vo_sort_t(tomo)
    srt = np.transpose(srt_t, (2, 1, 0))
    smooth = ndi.median_filter(srt, (1, 1, size))
    list1 = np.mean(srt[ndrop:nproj - ndrop], axis=0)
    list2 = np.mean(smooth[ndrop:nproj - ndrop], axis=0)
    fact = list1 / list2
    mask = _vo_dilate(_vo_detect(fact, snr))
    tomo = tomo / fact[None]
    corr = _vo_unsort_t(np.transpose(smooth, (2, 1, 0)), ids)
    np.copyto(tomo, corr, where=(mask[None] > 0.0))
    return tomo


def _vo_dead(tomo, snr, size):
    """_rs_dead3 (remove_stripe.py:427-454) on [nproj, nz, ni]: columns whose
    total variation along the angles stands out are replaced by linear
    interpolation between their unmasked neighbours, then _rs_large3."""
    import scipy.ndimage as ndi
    tomo = np.array(tomo, dtype=np.float32)
    nz = tomo.shape[1]
    smooth = ndi.uniform_filter1d(tomo, 10, axis=0)
    diff = np.sum(np.abs(tomo - smooth), axis=0)
    bck = ndi.median_filter(diff, (1, size))
    fact = diff / bck
    mask = _vo_dilate(_vo_detect(fact, snr))
    mask[:, 0:2] = 0.0
    mask[:, -2:] = 0.0
    for m in range(nz):
        good = np.where(mask[m] < 1.0)[0]
        miss = np.where(mask[m] > 0.0)[0]
        if len(miss) > 0:
            matz = tomo[:, m, good]
            ids = np.searchsorted(good, miss)
            tomo[:, m, miss] = (matz[:, ids - 1] + (miss - good[ids - 1]) *
                                (matz[:, ids] - matz[:, ids - 1]) / (good[ids] - good[ids - 1]))
    return _vo_large(tomo, snr, size)


def remove_all_stripe(tomo, snr=3, la_size=61, sm_size=21, dim=1):
    """remove_all_stripe (remove_stripe.py:457-498) on float32 [nproj, nz, ni]:
    dead and large stripes (_rs_dead3, window la_size), then small-to-medium
    stripes by a median of the angle-sorted values along the detector
    (_rs_sort3, window sm_size; dim 2 adds the window along the angles).
    Sorts along the angles are stable (CuPy's argsort is)."""
    import scipy.ndimage as ndi
    tomo = _vo_dead(tomo, snr, la_size)
    srt_t, ids = _vo_sort_t(tomo)
    srt_t = ndi.median_filter(srt_t, (sm_size, 1, 1) if dim == 1 else (sm_size, 1, sm_size))
    return _vo_unsort_t(srt_t, ids)


# --------------------------------------------------------------------------
# Fourier-wavelet ring removal (src/tomocupy/processing/remove_stripe.py:51-293)
# --------------------------------------------------------------------------
def _fw_sym_index(m1, length, m2):
    """Indices -m1 .. length+m2-1 folded into [0, length) by the half-sample
    symmetric reflection of _reflect/_mypad (remove_stripe.py:51-88)."""
    x = np.arange(-m1, length + m2)
    period = 2 * length
    r = np.mod(x, period)
    return np.where(r >= length, period - 1 - r, r)


def _fw_coeff_len(n, L):
    """pywt.dwt_coeff_len(n, L, 'symmetric') = floor((n + L - 1) / 2)."""
    return (n + L - 1) // 2


def _fw_analysis(x, lo, hi, axis):
    """afb1d (remove_stripe.py:90-126): symmetric pad, stride-2 correlation with
    the time-reversed taps, tap by tap in float32 (product, then sum: no
    fused multiply-add); returns (low, high) along ``axis`` (2 or 3)."""
    L = lo.size
    N = x.shape[axis]
    out = _fw_coeff_len(N, L)
    p = 2 * (out - 1) - N + L
    x = np.take(x, _fw_sym_index(p // 2, N, (p + 1) // 2), axis=axis)

    def tap(j):
        sl = [slice(None)] * 4
        sl[axis] = slice(j, j + 2 * out, 2)
        return x[tuple(sl)]
    a = lo[0] * tap(0)
    b = hi[0] * tap(0)
    for j in range(1, L):
        s = tap(j)
        a = a + lo[j] * s
        b = b + hi[j] * s
    return a.astype(np.float32), b.astype(np.float32)


def _fw_synthesis(lo, hi, g0, g1, axis):
    """sfb1d (remove_stripe.py:129-154): zero-initialised upsampled scatter of
    g0[j]*lo + g1[j]*hi at offsets j, j+2, ... then the crop of L-2 samples on
    each side, float32 throughout."""
    L = g0.size
    H = lo.shape[axis]
    full = (H - 1) * 2 + L
    shape = list(lo.shape)
    shape[axis] = full
    out = np.zeros(shape, dtype=np.float32)
    for j in range(L):
        sl = [slice(None)] * 4
        sl[axis] = slice(j, j + 2 * H, 2)
        out[tuple(sl)] += g0[j] * lo + g1[j] * hi
    sl = [slice(None)] * 4
    sl[axis] = slice(L - 2, full - (L - 2))
    return out[tuple(sl)]


def remove_stripe_fw(data, sigma, level, bank, fft=NumpyFFT):
    """remove_stripe_fw on float32 [nproj, nz, n] (returns a new array).

    ``bank`` = (dec_lo, dec_hi, rec_lo, rec_hi) of the wavelet (PyWavelets'
    filter-bank convention).  The sinogram stack is zero-padded along the
    angles to nproj + nproj//8 (centred), decomposed ``level`` times (rows
    along the detector first, then columns along the angles); at every level
    the band that is high-pass along the detector and low-pass along the
    angles is damped along the angles by 1 - exp(-y^2 / (2 sigma^2)) in the
    rfft domain; then the inverse transform and the crop.  Same float32
    operation order as the reference run with NumPy for CuPy."""
    dec_lo, dec_hi, rec_lo, rec_hi = (np.asarray(b, dtype=np.float64) for b in bank)
    h0 = dec_lo.astype(np.float32)[::-1].copy()
    h1 = dec_hi.astype(np.float32)[::-1].copy()
    g0 = rec_lo.astype(np.float32)
    g1 = rec_hi.astype(np.float32)
    data = np.asarray(data, dtype=np.float32)
    nproj, nz, ni = data.shape
    npad = nproj + nproj // 8
    sli = np.zeros((nz, 1, npad, ni), dtype=np.float32)
    sli[:, 0, (npad - nproj) // 2:(npad + nproj) // 2] = data.swapaxes(0, 1)
    bands = []
    for _ in range(level):
        rlo, rhi = _fw_analysis(sli, h0, h1, axis=3)     # along the detector
        ll, lh = _fw_analysis(rlo, h0, h1, axis=2)       # along the angles
        hl, hh = _fw_analysis(rhi, h0, h1, axis=2)
        # yh[:, 0, 0..2] = (low-row/high-col, high-row/low-col, high/high)
        band = hl[:, 0]
        my = band.shape[1]
        spec = fft.rfft(band, axis=1)
        yhat = np.fft.ifftshift((np.arange(-my, my, 2) + 1) / 2)[:my // 2 + 1]
        spec *= (-np.expm1(-yhat ** 2 / (2 * sigma ** 2)))[:, None]
        hl = fft.irfft(spec, my, axis=1).astype(np.float32)[:, None]
        bands.append((lh, hl, hh))
        sli = ll
    for lh, hl, hh in bands[::-1]:
        h, w = hl.shape[2], hl.shape[3]
        sli = sli[:, :, :h, :w]
        lo_hi = _fw_synthesis(np.concatenate([sli, hl], axis=1), np.concatenate([lh, hh], axis=1),
                              g0, g1, axis=2)
        sli = _fw_synthesis(lo_hi[:, :1], lo_hi[:, 1:], g0, g1, axis=3)
    out = sli[:, 0, (npad - nproj) // 2:(npad + nproj) // 2, :ni]
    return np.ascontiguousarray(out.swapaxes(0, 1)).astype(np.float32)


# --------------------------------------------------------------------------
# phase retrieval (src/tomocupy/processing/retrieve_phase.py:57-305)
# --------------------------------------------------------------------------
_PR_PLANCK = 6.58211928e-19   # retrieve_phase.py:45-48
_PR_LIGHT = 299792458e+2
_PR_PI = 3.14159265359


def pr_wavelength(energy):
    """_wavelength (retrieve_phase.py:51-52), cm."""
    return 2 * _PR_PI * _PR_PLANCK * _PR_LIGHT / energy


def pr_pads(dy, dz, pixel_size, dist, energy, pad=True):
    """(py, pz) of _calc_pad / _calc_pad_width (retrieve_phase.py:178-226)."""
    if not pad:
        return 0, 0
    wl = pr_wavelength(energy)

    def width(dim):
        pad_pix = np.ceil(_PR_PI * wl * dist / pixel_size ** 2)
        return int((pow(2, np.ceil(np.log2(dim + pad_pix))) - dim) * 0.5)
    return width(dy), width(dz)


def _pr_coord(pixel_size, num):
    """_reciprocal_coord (retrieve_phase.py:285-305), float32."""
    n = num - 1
    rc = np.arange(-n, num, 2, dtype=np.float32)
    rc *= 0.5 / (n * pixel_size)
    return rc


def pr_filter(method, ny, nz, pixel_size, dist, energy, alpha=1e-3, db=1000, W=2e-4):
    """The fftshifted filter of paganin_filter / farago_filter
    (retrieve_phase.py:85-93, 119-121, 209-258), float32 like the reference."""
    wl = pr_wavelength(energy)
    if method == "Gpaganin":
        ix = np.cos(_pr_coord(pixel_size, ny) * 2 * _PR_PI * pixel_size)
        iy = np.cos(_pr_coord(pixel_size, nz) * 2 * _PR_PI * pixel_size)
        a, b = np.meshgrid(iy, ix)
        kf = a + b
        aph = db * (dist * wl) / (4 * _PR_PI)
        f = 1 / (1.0 - (2 * aph / (W ** 2)) * (kf - 2))
    else:
        ix = np.square(_pr_coord(pixel_size, ny))
        iy = np.square(_pr_coord(pixel_size, nz))
        a, b = np.meshgrid(iy, ix)
        w2 = a + b
        if method == "paganin":
            f = 1 / (wl * dist * w2 / (4 * _PR_PI) + alpha)
        elif method == "farago":
            f = 1 / (np.cos(_PR_PI * wl * dist * w2) + db * np.sin(_PR_PI * wl * dist * w2))
        else:
            raise ValueError(method)
    return np.fft.fftshift(f).astype(np.float32)


def retrieve_phase(data, method, pixel_size=1e-4, dist=50, energy=20, alpha=1e-3, db=1000,
                   W=2e-4, pad=True):
    """paganin_filter / farago_filter on float32 projections [nproj, dy, dz]
    (retrieve_phase.py:57-145): edge padding by slice assignment, complex64
    fft2, the normalised filter, ifft2, real part, crop.  Returns a new array."""
    data = np.array(data, dtype=np.float32)
    nproj, dy, dz = data.shape
    px, py = pr_pads(dy, dz, pixel_size, dist, energy, pad)
    f = pr_filter(method, dy + 2 * px, dz + 2 * py, pixel_size, dist, energy, alpha, db, W)
    nf = f / f.max()
    prj = np.zeros((dy + 2 * px, dz + 2 * py), np.float32)
    for m in range(nproj):
        prj[px:dy + px, py:dz + py] = data[m]
        prj[:px] = prj[px]
        prj[-px:] = prj[-px - 1]        # px = 0: the whole array takes the last row
        prj[:, :py] = prj[:, py][:, np.newaxis]
        prj[:, -py:] = prj[:, -py - 1][:, np.newaxis]
        fproj = np.fft.fft2(prj.astype(np.complex64)).astype(np.complex64)
        fproj *= nf
        proj = np.real(np.fft.ifft2(fproj)).astype(np.float32)
        if pad:
            proj = proj[px:dy + px, py:dz + py]
        data[m] = proj
    return data


# --------------------------------------------------------------------------
# filter (reconstruction/fbp_filter.py:60-118, backproj_functions.py:93-109)
# --------------------------------------------------------------------------
def wint(n, t):
    N = len(t)
    s = np.linspace(1e-40, 1, n)
    iv = np.linalg.inv(np.exp(np.outer(np.arange(n), np.log(s))))
    k = np.arange(1, n + 2)
    u = np.diff(np.exp(np.outer(k, np.log(s))) * np.tile(1.0 / k[..., None], [1, n]))
    W1 = iv @ u[1:n + 1, :]
    W2 = iv @ u[0:n, :]
    p = 1 / np.concatenate((np.arange(1, n), (n - 1) * np.ones(N - 2 * (n - 1) - 1),
                            np.arange(n - 1, 0, -1)))
    w = np.zeros(N)
    for j in range(N - n + 1):
        W = ((t[j + n - 1] - t[j]) ** 2) * W1 + (t[j + n - 1] - t[j]) * t[j] * W2
        for kk in range(n - 1):
            w[j:j + n] = w[j:j + n] + p[j + kk] * W[:, kk]
    w[-40:] = (w[-40]) / (N - 40) * np.arange(N - 40, N)
    return w


def calc_filter(ne, name):
    d = 0.5
    t = np.arange(0, ne / 2 + 1) / ne
    windows = {
        "ramp": lambda: 1.0,
        "shepp": lambda: np.sinc(t / (2 * d)) * (t / d <= 2),
        "cosine": lambda: np.cos(np.pi * t / (2 * d)) * (t / d <= 1),
        "cosine2": lambda: (np.cos(np.pi * t / (2 * d))) ** 2 * (t / d <= 1),
        "hamming": lambda: (.54 + .46 * np.cos(np.pi * t / d)) * (t / d <= 1),
        "hann": lambda: (1 + np.cos(np.pi * t / d)) / 2.0 * (t / d <= 1),
        "parzen": lambda: pow(1 - t / d, 3) * (t / d <= 1),
    }
    if name == "none":
        wfa = ne * 0.5 + t * 0
        wfa[0] *= 2
    else:
        wfa = ne * 0.5 * wint(12, t) * windows[name]()
    wfa = 2 * wfa * (wfa >= 0)
    wfa[0] *= 2
    return wfa.astype("float32") / ne


def rfftfreq32(ne):
    return (np.arange(0, ne // 2 + 1, dtype=np.float64) / ne).astype(np.float32)


def phase_weights(wfilter, t, center, sht, n):
    """complex64 [nz, ne/2+1] in the reference's float32 operation order."""
    a = (np.float32(-center) + np.asarray(sht, np.float32)) + np.float32(n / 2)
    ci = np.float32(-2.0) * np.float32(math.pi)
    phase = (a * ci)[:, None] * t[None, :]
    return (wfilter * np.cos(phase) + 1j * (wfilter * np.sin(phase))).astype(np.complex64)


def filter_rows(rows, w, dtype=np.float32):
    """cfunc_filter::filter: R2C (len ne) -> * w[z] -> C2R (unnormalised)."""
    ne = rows.shape[-1]
    cdt = np.complex64 if dtype == np.float32 else np.complex128
    spec = sfft.rfft(rows.astype(dtype), axis=-1, workers=WORKERS).astype(cdt)
    spec *= w.astype(cdt)[:, None, :]
    return sfft.irfft(spec, n=ne, axis=-1, norm="forward", workers=WORKERS).astype(dtype)


def fbp_filter_center(data, wfilter, center, sht, dtype=np.float32):
    """Edge pad [nz, P, n] rows to ne, filter with the centred spectra, crop back."""
    nz, nproj, n = data.shape
    ne = (len(wfilter) - 1) * 2
    pad = ne // 2 - n // 2
    rows = np.empty((nz, nproj, ne), dtype=dtype)
    rows[:, :, pad:pad + n] = data
    rows[:, :, :pad] = data[:, :, :1]
    rows[:, :, pad + n:] = data[:, :, -1:]
    w = phase_weights(wfilter, rfftfreq32(ne), center, np.broadcast_to(sht, (nz,)), n)
    if dtype == np.float64:
        w = _phase_weights64(wfilter, ne, center, np.broadcast_to(sht, (nz,)), n)
    out = filter_rows(rows, w, dtype)
    return np.ascontiguousarray(out[:, :, pad:pad + n])


def _phase_weights64(wfilter, ne, center, sht, n):
    t = np.arange(0, ne // 2 + 1, dtype=np.float64) / ne
    a = -center + np.asarray(sht, np.float64) + n / 2
    return wfilter.astype(np.float64) * np.exp(-2j * np.pi * a[:, None] * t[None, :])


# --------------------------------------------------------------------------
# fourierrec (src/include/kernels_fourierrec.cuh, src/cuda/cfunc_fourierrec.cu)
# --------------------------------------------------------------------------
def fourierrec_constants(n):
    eps = np.float32(1e-3)
    mu = np.float32(-np.log(eps)) / np.float32(2 * n * n)
    m = int(np.ceil(2 * n * 1 / np.float32(3.1415926535) *
                    np.sqrt(-mu * np.log(eps) + (mu * n) * (mu * n) / 4)))
    return mu, m


def fourierrec_pairs(gc, theta, n, dtype=np.float32):
    """cfunc_fourierrec::backprojection on complex pairs gc [nz, P, n] -> [nz, n, n]."""
    cdt = np.complex64 if dtype == np.float32 else np.complex128
    nz, nproj, _ = gc.shape
    mu, m = fourierrec_constants(n)
    mu = dtype(mu)
    pi = dtype(3.1415926535) if dtype == np.float32 else np.pi
    # takexy (kernels_fourierrec.cuh:23-36)
    th = np.asarray(theta, dtype=dtype)
    r = ((np.arange(n) - n // 2) / dtype(n)).astype(dtype)
    x = (r[None, :] * np.cos(th)[:, None]).astype(dtype)
    y = (-(r[None, :] * np.sin(th)[:, None])).astype(dtype)
    x[x >= 0.5] = dtype(0.5 - 1e-5)
    y[y >= 0.5] = dtype(0.5 - 1e-5)
    # ifftshiftc -> FFT(n) -> ifftshiftc
    sgn = (1 - 2 * ((np.arange(n) + 1) % 2)).astype(dtype)
    g = gc.astype(cdt) * sgn
    g = sfft.fft(g, axis=-1, workers=WORKERS).astype(cdt) * sgn
    # gather (kernels_fourierrec.cuh:60-119) with bincount accumulation
    N2 = 2 * n + 2 * m
    coeff0 = pi / (mu * dtype(4 * n * n))
    coeff1 = -pi * pi / mu
    b0 = np.floor(dtype(2 * n) * x).astype(np.int64) - m
    b1 = np.floor(dtype(2 * n) * y).astype(np.int64) - m
    k0 = [np.exp(coeff1 * ((b0 + i).astype(dtype) / dtype(2 * n) - x) ** 2).astype(dtype)
          for i in range(2 * m + 1)]
    k1 = [np.exp(coeff1 * ((b1 + i).astype(dtype) / dtype(2 * n) - y) ** 2).astype(dtype)
          for i in range(2 * m + 1)]
    fde = np.zeros((nz, N2 * N2), dtype=cdt)
    for z in range(nz):
        g0 = (g[z] * dtype(4.0 / n)).astype(cdt)
        acc_r = np.zeros(N2 * N2, dtype=np.float64)
        acc_i = np.zeros(N2 * N2, dtype=np.float64)
        for i1 in range(2 * m + 1):
            row = (n + m + b1 + i1) * N2
            for i0 in range(2 * m + 1):
                w = coeff0 * (k0[i0] * k1[i1])
                idx = (row + n + m + b0 + i0).ravel()
                acc_r += np.bincount(idx, weights=(w * g0.real).ravel(), minlength=N2 * N2)
                acc_i += np.bincount(idx, weights=(w * g0.imag).ravel(), minlength=N2 * N2)
        fde[z] = (acc_r + 1j * acc_i).astype(cdt)
    fde = fde.reshape(nz, N2, N2)
    # wrap (kernels_fourierrec.cuh:38-58): halo folded periodically
    core = fde[:, m:2 * n + m, m:2 * n + m].copy()
    tx = np.arange(N2)
    halo = (tx < m) | (tx >= 2 * n + m)
    dst = (tx - m + 2 * n) % (2 * n)
    ys, xs = np.nonzero(halo[:, None] | halo[None, :])
    for z in range(nz):
        np.add.at(core[z], (dst[ys], dst[xs]), fde[z, ys, xs])
    # fftshiftc over the (2n+2m)^2 buffer restricted to the interior, 2D inverse FFT
    idx = np.arange(m, 2 * n + m)
    s1 = (1 - 2 * ((idx + 1) % 2)).astype(dtype)
    sgn2 = s1[:, None] * s1[None, :]
    core = sfft.ifft2(core * sgn2, axes=(-2, -1), norm="forward", workers=WORKERS).astype(cdt)
    core = core * sgn2
    # divphi (kernels_fourierrec.cuh:4-21) + circ (:161-174)
    t = np.arange(n)
    dx = (t / dtype(n) - dtype(0.5)).astype(dtype)
    phi = np.exp(mu * dtype(n * n) * (dx[None, :] ** 2 + dx[:, None] ** 2)) / dtype(nproj)
    phi = phi * dtype(1 - n % 4)
    ix = t + n // 2
    iy = t + 1 + n // 2
    f = core[:, iy][:, :, ix] * phi.astype(dtype)
    xc = ((t - n // 2) / dtype(n)).astype(dtype)
    lam = ((4 * xc[None, :] ** 2 + 4 * xc[:, None] ** 2) < 1).astype(dtype)
    return (f * lam).astype(cdt)


def fourierrec(data, theta, dtype=np.float32):
    """FourierRec.backprojection (fourierrec.py:61-68): real [nz, P, n] -> [nz, n, n]."""
    nz, nproj, n = data.shape
    h = nz // 2
    gc = data[:h].astype(dtype) + 1j * data[h:].astype(dtype)
    f = fourierrec_pairs(gc, theta, n, dtype)
    return np.concatenate((f.real, f.imag)).astype(dtype)


# --------------------------------------------------------------------------
# linerec (src/include/kernels_linerec.cuh:3-137)
# --------------------------------------------------------------------------
def linerec(data, theta, n, nz, ncz, phi=np.pi / 2, sz=0, nproj_scale=None, sh=None,
            phis=None, dtype=np.float32):
    """f[ncz, n, n] = sum over angles of bilinear samples of data [nz, P, n]."""
    nproj = data.shape[1]
    c = dtype(4.0) / dtype(nproj_scale or nproj)
    tx = np.arange(n)
    X = (tx - n // 2).astype(dtype)[None, :]
    Y = (tx - n // 2).astype(dtype)[:, None]
    out = np.zeros((ncz, n, n), dtype=dtype)
    flat = data.astype(dtype).ravel()
    for tz in range(ncz):
        ph = dtype(phis[tz]) if phis is not None else dtype(phi)
        cphi, sphi = dtype(np.cos(ph)), dtype(np.sin(ph))
        zz = (tz + sz - nz // 2) if (sh is None and phis is None) else (sz - nz // 2)
        acc = np.zeros((n, n), dtype=dtype)
        for t in range(nproj):
            ct, st = dtype(np.cos(dtype(theta[t]))), dtype(np.sin(dtype(theta[t])))
            u = ct * X + st * Y + dtype(n // 2)
            if sh is not None:
                u = u - dtype(sh[tz])
            v = (st * cphi) * X + (-ct * cphi) * Y + sphi * dtype(zz) + dtype(nz // 2)
            u = np.broadcast_to(u, (n, n))
            v = np.broadcast_to(v, (n, n))
            ur = np.trunc(u - dtype(1e-5)).astype(np.int64)
            vr = np.trunc(v - dtype(1e-5)).astype(np.int64)
            ok = (ur >= 0) & (ur < n - 1) & (vr >= 0) & (vr < nz - 1)
            uu = np.where(ok, u - ur, 0).astype(dtype)
            vv = np.where(ok, v - vr, 0).astype(dtype)
            urc = np.where(ok, ur, 0)
            vrc = np.where(ok, vr, 0)
            base = urc + t * n + vrc * n * nproj
            val = (flat[base] * ((1 - uu) * (1 - vv)) + flat[base + 1] * (uu * (1 - vv)) +
                   flat[base + n * nproj] * ((1 - uu) * vv) +
                   flat[base + n * nproj + 1] * (uu * vv))
            acc += np.where(ok, val, 0).astype(dtype)
        out[tz] = (acc * c)[::-1]
    return out


def direct_fbp64(filtered, theta, n):
    """Direct FP64 pixel-driven backprojection with linear interpolation (discretisation
    truth for the filtered sinograms [nz, P, n]); same output orientation as fourierrec."""
    nz, nproj, _ = filtered.shape
    t = np.arange(n) - n / 2
    X, Y = np.meshgrid(t, t)
    out = np.zeros((nz, n, n))
    for p in range(nproj):
        s = X * np.cos(theta[p]) - Y * np.sin(theta[p]) + n / 2
        i0 = np.floor(s).astype(np.int64)
        fr = s - i0
        ok = (i0 >= 0) & (i0 < n - 1)
        i0c = np.clip(i0, 0, n - 2)
        for z in range(nz):
            row = filtered[z, p].astype(np.float64)
            out[z] += np.where(ok, row[i0c] * (1 - fr) + row[i0c + 1] * fr, 0)
    return out * np.pi / nproj


# --------------------------------------------------------------------------
# laminography Fourier chain in float64 (src/cuda/cfunc_fft2d.cu:52-63,
# src/include/kernels_fft2d.cu, src/cuda/cfunc_usfft2d.cu:72-89 with
# src/include/kernels_usfft2d.cu, src/cuda/cfunc_usfft1d.cu:68-86 with
# src/include/kernels_usfft1d.cu, glue of
# src/tomocupy/reconstruction/backproj_lamfourier_parallel.py:185-304).
# The frequency-row chunk packing of the glue is replaced by its meaning:
# row r of the half spectrum, with the conjugate mirror for tx > detw/2.
# --------------------------------------------------------------------------
def _usfft_params(n, eps=1e-3):
    mu = -np.log(eps) / (2.0 * n * n)
    m = int(np.ceil(2 * n / np.pi * np.sqrt(-mu * np.log(eps) + (mu * n) * (mu * n) / 4)))
    return mu, m


def _checker(nx, ny):
    """(1-2((tx+1)%2)) (1-2((ty+1)%2)) over [ny, nx]."""
    sx = 1 - 2 * ((np.arange(nx) + 1) % 2)
    sy = 1 - 2 * ((np.arange(ny) + 1) % 2)
    return (sy[:, None] * sx[None, :]).astype(np.float64)


def fft2d64(f):
    """cfunc_fft2d.fwd: sign flip, R2C 2D, sign flip with -1, / (deth*detw)."""
    ntheta, deth, detw = f.shape
    g = np.fft.rfft2(f * _checker(detw, deth)[None])
    wc = detw // 2 + 1
    return g * (-_checker(wc, deth))[None] / (deth * detw)


def usfft2d_adj64(s1, theta, phi, n):
    """All frequency rows r in [0, deth/2] of the half spectrum s1
    [ntheta, deth, detw/2+1] -> s2 [n1 = n, nrow, n0 = n] (usfft2d.adj)."""
    ntheta, deth, wc = s1.shape
    detw = 2 * (wc - 1)
    n0 = n1 = n
    mu0, m0 = _usfft_params(n0)
    mu1, m1 = _usfft_params(n1)
    P0, P1 = 2 * n0 + 2 * m0, 2 * n1 + 2 * m1
    nrow = deth // 2 + 1
    out = np.empty((n1, nrow, n0), dtype=np.complex128)
    th = np.asarray(theta, np.float64)[:, None]
    tx = np.arange(detw)[None, :]
    ku = (tx - detw / 2.0) / detw
    i0 = np.arange(2 * m0 + 1)
    i1 = np.arange(2 * m1 + 1)
    for r in range(nrow):
        kv = (r - deth / 2.0) / deth
        x = ku * np.cos(th) + kv * np.sin(th) * np.cos(phi)
        y = ku * np.sin(th) - kv * np.cos(th) * np.cos(phi)
        x = np.clip(x, -0.5 + 1e-5, 0.5 - 1e-5).ravel()
        y = np.clip(y, -0.5 + 1e-5, 0.5 - 1e-5).ravel()
        # sample values with the conjugate mirror of gather2d
        mrow = (deth - r) % deth
        v = np.where(tx <= detw // 2, s1[:, r, np.minimum(tx, wc - 1)[0]],
                     np.conj(s1[:, mrow, np.clip(detw - tx, 0, wc - 1)[0]])).ravel()
        ell0 = np.floor(2 * n0 * x).astype(np.int64)[:, None] - m0 + i0[None, :]
        ell1 = np.floor(2 * n1 * y).astype(np.int64)[:, None] - m1 + i1[None, :]
        w0 = ell0 / (2.0 * n0) - x[:, None]
        w1 = ell1 / (2.0 * n1) - y[:, None]
        w = (np.pi / np.sqrt(mu0 * mu1 * ntheta) *
             np.exp(-np.pi ** 2 / mu0 * w0[:, None, :] ** 2 - np.pi ** 2 / mu1 * w1[:, :, None] ** 2))
        idx = (n0 + m0 + ell0[:, None, :]) + P0 * (n1 + m1 + ell1[:, :, None])
        val = (w * v[:, None, None]).ravel()
        idx = idx.ravel()
        grid = (np.bincount(idx, val.real, P0 * P1) + 1j * np.bincount(idx, val.imag, P0 * P1))
        grid = grid.reshape(P1, P0)
        # wrap2d (adjoint): fold the padding into the periodic 2n grid
        core = np.zeros((2 * n1, 2 * n0), dtype=np.complex128)
        yy = (np.arange(P1) - m1) % (2 * n1)
        xx = (np.arange(P0) - m0) % (2 * n0)
        np.add.at(core, (yy[:, None], xx[None, :]), grid)
        grid = np.zeros((P1, P0), dtype=np.complex128)
        grid[m1:m1 + 2 * n1, m0:m0 + 2 * n0] = core
        grid *= _checker(P0, P1)
        inner = grid[m1:m1 + 2 * n1, m0:m0 + 2 * n0]
        grid[m1:m1 + 2 * n1, m0:m0 + 2 * n0] = np.fft.ifft2(inner) * (4 * n0 * n1)
        grid *= _checker(P0, P1)
        # divker2d (direction 1): f[ty][slab][tx] with the n1-ty-1 row flip
        ty = np.arange(n1)[:, None]
        txo = np.arange(n0)[None, :]
        ker = np.exp(-mu0 * (txo - n0 // 2) ** 2 - mu1 * (ty - n1 // 2) ** 2)
        gv = grid[n1 - ty - 1 + n1 // 2 + m1, txo + n0 // 2 + m0]
        out[:, r, :] = gv / ker / (n0 * n1)
    return out


def usfft1d_adj64(s2, phi, rh, deth):
    """s2 [n1, deth/2+1, n0] -> f [n1, rh, n0] real (usfft1d.adj along the height)."""
    n1, hc, n0 = s2.shape
    n2 = rh
    mu2, m2 = _usfft_params(n2)
    P2 = 2 * n2 + 2 * m2
    tz = np.arange(deth)
    z = (tz - deth / 2.0) / deth * np.sin(phi)
    tzs = np.where(tz > deth // 2, deth - tz, tz)
    conj = np.where(tz > deth // 2, -1.0, 1.0)
    g = s2[:, tzs, :]                                  # [n1, deth, n0]
    g = g.real + 1j * (g.imag * conj[None, :, None])
    i2 = np.arange(2 * m2 + 1)
    ell2 = np.floor(2 * n2 * z).astype(np.int64)[:, None] - m2 + i2[None, :]   # [deth, 2m2+1]
    w = np.sqrt(np.pi / (mu2 * n0)) * np.exp(-np.pi ** 2 / mu2 * (ell2 / (2.0 * n2) - z[:, None]) ** 2)
    grid = np.zeros((n1, P2, n0), dtype=np.complex128)
    for t in range(deth):
        for j in range(2 * m2 + 1):
            grid[:, n2 + m2 + ell2[t, j], :] += w[t, j] * g[:, t, :]
    core = np.zeros((n1, 2 * n2, n0), dtype=np.complex128)
    zz = (np.arange(P2) - m2) % (2 * n2)
    for k in range(P2):
        core[:, zz[k], :] += grid[:, k, :]
    grid[:] = 0
    grid[:, m2:m2 + 2 * n2, :] = core
    s = (1 - 2 * ((np.arange(P2) + 1) % 2)).astype(np.float64)[None, :, None]
    grid *= s
    grid[:, m2:m2 + 2 * n2, :] = np.fft.ifft(grid[:, m2:m2 + 2 * n2, :], axis=1) * (2 * n2)
    grid *= s
    tzo = np.arange(n2)
    ker = np.exp(-mu2 * (tzo - n2 // 2) ** 2)
    return grid[:, tzo + n2 // 2 + m2, :].real / ker[None, :, None] / (2 * n2)


def rec_lam64(data, theta, center, lamino_angle, rh, wfilter):
    """FP64 laminographic reconstruction [rh, detw, detw] of data [ntheta, deth, detw]."""
    ntheta, deth, detw = data.shape
    phi = np.pi / 2 + lamino_angle / 180 * np.pi
    filt = fbp_filter_center(np.asarray(data, np.float64), wfilter, center, 0.0, np.float64)
    s1 = fft2d64(filt)
    s2 = usfft2d_adj64(s1, theta, phi, detw)
    s3 = usfft1d_adj64(s2, phi, rh, deth)
    return np.ascontiguousarray(s3.transpose(1, 0, 2))


# ---------------------------------------------------------------- rotation
def rotate_params(angle, nz, n):
    """(c, s, offz, offx) of ndimage.rotate(angle, axes=(2, 1), reshape=False)
    on nz x n planes, as the reference's host code forms them
    (src/tomocupy/processing/proc_functions.py:126-138 calls cupyx's rotate,
    which builds the matrix from NumPy's deg2rad, cos and sin)."""
    a = np.deg2rad(float(angle))
    c, s = float(np.cos(a)), float(np.sin(a))
    rot = np.array([[c, s], [-s, c]])
    shape = np.array([nz, n], dtype=np.float64)
    off = (shape - 1) / 2 - rot @ ((shape - 1) / 2)
    return c, s, float(off[0]), float(off[1])


def rotate_planes(data, c, s, offz, offx, order=1):
    """The geometric transform of scipy.ndimage (its published algorithm,
    restated for spline orders 0 and 1, mode 'nearest'): every output pixel
    (oz, ox) of each [nz, n] plane of data [k, nz, n] samples the input at
    iz = (offz + oz c) + ox s, ix = (offx + oz (-s)) + ox c, clamped to
    [0, len - 1]; order 1 weights (1 - t, 1 - (1 - t)); terms v * wz * wx
    summed from 0 in the order (z0,x0), (z0,x1), (z1,x0), (z1,x1); float64
    rounded to float32 once."""
    data = np.asarray(data, dtype=np.float32)
    k, nz, n = data.shape
    oz = np.arange(nz, dtype=np.float64)[:, None]
    ox = np.arange(n, dtype=np.float64)[None, :]
    iz = (offz + oz * c) + ox * s
    ix = (offx + oz * (-s)) + ox * c
    iz = np.clip(iz, 0.0, nz - 1.0)
    ix = np.clip(ix, 0.0, n - 1.0)
    d = data.astype(np.float64)
    if order == 0:
        z0 = np.minimum(np.floor(iz + 0.5).astype(np.int64), nz - 1)
        x0 = np.minimum(np.floor(ix + 0.5).astype(np.int64), n - 1)
        return d[:, z0, x0].astype(np.float32)
    if order != 1:
        raise NotImplementedError("spline orders 0 and 1")
    fz, fx = np.floor(iz), np.floor(ix)
    z0, x0 = fz.astype(np.int64), fx.astype(np.int64)
    z1, x1 = np.minimum(z0 + 1, nz - 1), np.minimum(x0 + 1, n - 1)
    wz0 = 1.0 - (iz - fz)
    wz1 = 1.0 - wz0
    wx0 = 1.0 - (ix - fx)
    wx1 = 1.0 - wx0
    v = np.zeros((k, nz, n), dtype=np.float64)
    v = v + d[:, z0, x0] * wz0 * wx0
    v = v + d[:, z0, x1] * wz0 * wx1
    v = v + d[:, z1, x0] * wz1 * wx0
    v = v + d[:, z1, x1] * wz1 * wx1
    return v.astype(np.float32)


def rotate_proj(data, angle, order=1):
    """ProcFunctions.rotate_proj (proc_functions.py:126-138) of [nproj, nz, n]."""
    _, nz, n = np.shape(data)
    return rotate_planes(data, *rotate_params(angle, nz, n), order=order)
