"""Pre-processing of projection chunks.

``ProcFunctions`` mirrors the reference class
(src/tomocupy/processing/proc_functions.py:47-198) for the hot-path steps:
``darkflat_correction`` and ``minus_log`` run as native kernels with the
reference's float32 operation order (bit-identical results), and so do
``remove_outliers`` (dezinger: a [w, 1, w] median, bit-identical on integer
frames) and the phase-retrieval, rotation and double-FOV padding steps of
``proc_proj``.  Beam hardening is outside this package's scope and raises
``NotImplementedError`` when enabled, instead of silently doing nothing.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _lib
from ..global_vars import args, params

_DT = {torch.uint16: _lib.TCB_U16, torch.uint8: _lib.TCB_U8, torch.float32: _lib.TCB_F32}


def in_dtype_code(t: torch.Tensor) -> int:
    try:
        return _DT[t.dtype]
    except KeyError:
        raise TypeError(f"unsupported frame dtype {t.dtype}; expected uint16, uint8 or float32")


def dezinger(frames: torch.Tensor, width: int, threshold: float, out=None,
             stream=None) -> torch.Tensor:
    """remove_outliers of frames [k, nz, n] (proc_functions.py:96-107) into a new
    contiguous tensor (or ``out``): median over width frames x width columns of a
    row, mode 'reflect', replacing pixels more than ``threshold`` above it.  The
    input may be a view whose rows are contiguous."""
    k, nz, n = frames.shape
    if frames.stride(2) != 1:
        raise ValueError("dezinger: rows must be contiguous")
    if out is None:
        out = torch.empty((k, nz, n), dtype=frames.dtype, device=frames.device)
    assert out.is_contiguous() and out.shape == frames.shape and out.dtype == frames.dtype
    _lib.call("tcb_dezinger", _lib.ptr(out), _lib.ptr(frames), in_dtype_code(frames), k, nz, n,
              frames.stride(0), frames.stride(1), int(width), float(threshold),
              _lib.stream_ptr(stream))
    return out


def downsample(frames: torch.Tensor, binning: int, out=None, stream=None) -> torch.Tensor:
    """utils.downsample (src/tomocupy/utils.py:157-167) of float32-converted
    frames [k, nz * 2^b, n * 2^b] (device; any dtype of uint8 / uint16 /
    float32, rows contiguous) -> float32 [k, nz, n] block sums, columns then
    rows as pairwise trees."""
    k, zr, nr = frames.shape
    b = int(binning)
    nz, n = zr >> b, nr >> b
    if frames.stride(2) != 1:
        raise ValueError("downsample: rows must be contiguous")
    if out is None:
        out = torch.empty((k, nz, n), dtype=torch.float32, device=frames.device)
    _lib.call("tcb_downsample", _lib.ptr(out), _lib.ptr(frames), in_dtype_code(frames), k, nz, n,
              frames.stride(0), frames.stride(1), b, _lib.stream_ptr(stream))
    return out


def rotate_params(angle: float, nz: int, n: int):
    """(c, s, offz, offx) of ndimage.rotate(angle, axes=(2, 1), reshape=False)
    on planes of nz x n, computed as the reference's cupyx call does on the
    host: NumPy float64 deg2rad, cos, sin, and the offset that maps the
    rotated plane centre onto the input's."""
    a = np.deg2rad(float(angle))
    c, s = float(np.cos(a)), float(np.sin(a))
    rot = np.array([[c, s], [-s, c]])
    shape = np.array([nz, n], dtype=np.float64)
    off = (shape - 1) / 2 - rot @ ((shape - 1) / 2)
    return c, s, float(off[0]), float(off[1])


def rotate_proj(data: torch.Tensor, angle: float, order: int = 1, out=None,
                stream=None) -> torch.Tensor:
    """ProcFunctions.rotate_proj (proc_functions.py:126-138): every projection
    of float32 data [nproj, nz, n] (device, rows contiguous) rotated by angle
    degrees about its centre, ndimage.rotate(reshape=False, order,
    axes=(2, 1), mode='nearest'); spline orders 0 and 1.  Returns a new
    tensor (or out, which must not overlap data)."""
    nproj, nz, n = data.shape
    if data.dtype != torch.float32 or data.stride(2) != 1 or data.stride(1) != n:
        raise ValueError("rotate_proj: float32 frames with contiguous rows of n samples")
    if int(order) not in (0, 1):
        raise NotImplementedError(f"rotate_proj: spline order {order} (orders 0 and 1)")
    if out is None:
        out = torch.empty((nproj, nz, n), dtype=torch.float32, device=data.device)
    c, s, offz, offx = rotate_params(angle, nz, n)
    _lib.call("tcb_rotate_proj", _lib.ptr(out), _lib.ptr(data), nproj, nz, n, data.stride(0),
              out.stride(0), c, s, offz, offx, int(order), _lib.stream_ptr(stream))
    return out


def pad360_args():
    """(flip, w) of pad360 (proc_functions.py:109-124) for a double-FOV scan, else None."""
    if args.file_type != "double_fov":
        return None
    flip = params.centeri < params.ni // 2
    return flip, max(1, int(2 * (params.ni - params.center)))


def pad360(data: torch.Tensor, flip: bool, w: int) -> torch.Tensor:
    """ProcFunctions.pad360 (proc_functions.py:109-124): float32 [nproj, nz, ni]
    -> [nproj, nz, 2 ni], each row optionally flipped, its last w samples
    times the smooth transition, zero-padded."""
    import ctypes as C
    nproj, nz, ni = data.shape
    v = np.empty(int(w), dtype=np.float64)
    _lib.call("tcb_pad360_weights", v.ctypes.data_as(C.c_void_p), int(w))
    vd = torch.as_tensor(v, device=data.device)
    padded = torch.empty((nproj, nz, 2 * ni), dtype=torch.float32, device=data.device)
    padded[:, :, :ni] = data
    _lib.call("tcb_pad360_rows", padded.data_ptr(), nproj * nz, ni, 2 * ni, int(flip),
              vd.data_ptr(), int(w), _lib.stream_ptr(None))
    return padded


def dezinger_args():
    """(width, threshold) when args.dezinger enables outlier removal, else None."""
    w = int(args.dezinger)
    return (w, float(args.dezinger_threshold)) if w > 0 else None


def darkflat_stats(dark: torch.Tensor, flat: torch.Tensor, bright_ratio: float = 1.0,
                   flat_linear: bool = False, stream=None):
    """dark0 [nz, n], flat0 [nz, n] (and flat1 for flat_linear) from [k, nz, n] frames."""
    nd, nz, n = dark.shape
    nf = flat.shape[0]
    assert flat.shape[1:] == (nz, n), "dark/flat shapes differ"
    assert dark.dtype == flat.dtype
    dark = dark.contiguous()
    flat = flat.contiguous()
    dev = dark.device
    dark0 = torch.empty((nz, n), dtype=torch.float32, device=dev)
    flat0 = torch.empty((nz, n), dtype=torch.float32, device=dev)
    flat1 = torch.empty((nz, n), dtype=torch.float32, device=dev) if flat_linear else None
    _lib.call("tcb_darkflat_stats", _lib.ptr(dark0), _lib.ptr(flat0), _lib.ptr(flat1),
              _lib.ptr(dark), _lib.ptr(flat), nd, nf, nz, n, in_dtype_code(dark),
              float(bright_ratio), int(flat_linear), _lib.stream_ptr(stream))
    return dark0, flat0, flat1


def prep_rows(out, data, dark0=None, flat0=None, flat1=None, *, darkflat=True, minus_log=True,
              flat_linear=False, out_zstride, out_pstride, out_poff=0, out_xoff=0,
              out_width=None, edge_pad=False, stream=None):
    """Fused native pass over rows of a [nproj, nz, n] stack (see tcb_prep_rows)."""
    nproj, nz, n = data.shape
    assert data.stride(2) == 1
    flags = 0
    if darkflat:
        flags |= _lib.PREP_DARKFLAT
    if minus_log:
        flags |= _lib.PREP_MINUS_LOG
    if flat_linear:
        flags |= _lib.PREP_FLAT_LINEAR
    if edge_pad:
        flags |= _lib.PREP_EDGE_PAD
    _lib.call("tcb_prep_rows", _lib.ptr(out), _lib.ptr(data), _lib.ptr(dark0), _lib.ptr(flat0),
              _lib.ptr(flat1), nproj, nz, n, data.stride(0), data.stride(1), in_dtype_code(data),
              out_zstride, out_pstride, out_poff, out_xoff,
              out_width if out_width is not None else out_xoff + n, flags,
              _lib.stream_ptr(stream))
    return out


def prep_rows_split16(hi, lo, data, dark0=None, flat0=None, flat1=None, *, darkflat=True,
                      minus_log=True, flat_linear=False, out_zstride, out_pstride,
                      stream=None):
    """tcb_prep_rows_split16: the prep_rows chain written as fp16 hi/lo planes."""
    nproj, nz, n = data.shape
    assert data.stride(2) == 1
    assert hi.dtype == torch.float16 and lo.dtype == torch.float16
    flags = 0
    if darkflat:
        flags |= _lib.PREP_DARKFLAT
    if minus_log:
        flags |= _lib.PREP_MINUS_LOG
    if flat_linear:
        flags |= _lib.PREP_FLAT_LINEAR
    _lib.call("tcb_prep_rows_split16", _lib.ptr(hi), _lib.ptr(lo), _lib.ptr(data),
              _lib.ptr(dark0), _lib.ptr(flat0), _lib.ptr(flat1), nproj, nz, n, data.stride(0),
              data.stride(1), in_dtype_code(data), out_zstride, out_pstride, flags,
              _lib.stream_ptr(stream))
    return hi, lo


PHASE_METHODS = ("paganin", "Gpaganin", "farago")


def retrieve_phase(data):
    """The phase-retrieval step of proc_proj (proc_functions.py:169-181), in
    place on float32 projections [nproj, dy, dz] on the device, with the
    reference's unit conversions (pixel_size um -> cm, propagation_distance
    mm -> cm, W um -> cm).  'FourierFilter', a config choice that the
    reference's proc_proj never matches (it tests for 'FF'), does nothing
    there and does nothing here."""
    method = args.retrieve_phase_method
    if method in ("none", "FourierFilter"):
        return data
    if method not in PHASE_METHODS:
        raise NotImplementedError(f"retrieve_phase_method={method!r}")
    from . import retrieve_phase as rp
    data = data.contiguous()
    ps, dist = args.pixel_size * 1e-4, args.propagation_distance / 10
    if method == "farago":
        return rp.farago_filter(data, ps, dist, args.energy, args.retrieve_phase_delta_beta,
                                method)
    return rp.paganin_filter(data, ps, dist, args.energy, args.retrieve_phase_alpha, method,
                             args.retrieve_phase_delta_beta, args.retrieve_phase_W * 1e-4)


class ProcFunctions:
    def __init__(self):
        if args.beam_hardening_method != "none":
            raise NotImplementedError("beam hardening is not part of tomocupy_b200")

    def darkflat_correction(self, data, dark, flat):
        """(data - mean(dark)) / (mean(flat/bright_ratio)*(1+1e-5) - mean(dark)), float32."""
        flat_linear = args.flat_linear == "True" and data.shape[0] == params.nproj
        dark0, flat0, flat1 = darkflat_stats(dark, flat, args.bright_ratio, flat_linear)
        nproj, nz, n = data.shape
        res = torch.empty((nproj, nz, n), dtype=torch.float32, device=data.device)
        prep_rows(res, data, dark0, flat0, flat1, darkflat=True, minus_log=False,
                  flat_linear=flat_linear, out_zstride=n, out_pstride=nz * n)
        return res

    def minus_log(self, data):
        """In place: where(x<=0,1,x) -> -log -> nan_to_num(nan=6, posinf=0, neginf=0)."""
        assert data.dtype == torch.float32 and data.is_contiguous()
        nproj, nz, n = data.shape
        prep_rows(data, data, darkflat=False, minus_log=True, out_zstride=n,
                  out_pstride=nz * n)
        return data

    def remove_outliers(self, data):
        """In place, like the reference's data[:] = remove_outliers(data)."""
        dz = dezinger_args()
        if dz is not None:
            data.copy_(dezinger(data, *dz))
        return data

    def proc_sino(self, data, dark, flat, res=None):
        """Processing of a sinogram chunk: dark/flat correction and ring removal."""
        data = self.remove_outliers(data)
        dark = self.remove_outliers(dark)
        flat = self.remove_outliers(flat)
        out = self.darkflat_correction(data, dark, flat)
        if args.remove_stripe_method == "fw":
            from . import remove_stripe
            out = remove_stripe.remove_stripe_fw(out, args.fw_sigma, args.fw_filter,
                                                 args.fw_level)
        elif args.remove_stripe_method == "ti":
            from . import remove_stripe
            out = remove_stripe.remove_stripe_ti(out, args.ti_beta, args.ti_mask)
        elif args.remove_stripe_method != "none":
            raise NotImplementedError(
                f"remove_stripe_method={args.remove_stripe_method!r} is not part of tomocupy_b200")
        if res is not None:
            res[:] = out
            return res
        return out

    def rotate_proj(self, data, angle, order=2):
        """In place, like the reference's data[:] = ndimage.rotate(...)."""
        data.copy_(rotate_proj(data.contiguous(), angle, order))
        return data

    def pad360(self, data):
        """[nproj, nz, ni] -> [nproj, nz, 2 ni] for a double-FOV scan."""
        return pad360(data.contiguous(), *pad360_args())

    def proc_proj(self, data, st=None, end=None, res=None):
        """Processing of a projection chunk (proc_functions.py:163-196): phase
        retrieval, rotation, -log, double-FOV padding (beam hardening is out
        of scope)."""
        data = retrieve_phase(data)
        if float(args.rotate_proj_angle) != 0:
            data = self.rotate_proj(data.contiguous(), args.rotate_proj_angle,
                                    args.rotate_proj_order)
        if args.minus_log == "True":
            data = self.minus_log(data.contiguous())
        if args.file_type == "double_fov":
            data = self.pad360(data)
        if res is not None:
            res[:] = data
            return res
        return data
