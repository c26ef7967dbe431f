"""Fourier-wavelet (``remove_stripe_fw``), Titarenko (``remove_stripe_ti``) and
Vo's all-stripe (``remove_all_stripe``) ring removal over the native operators.

Same function signature and result layout as the reference
(src/tomocupy/processing/remove_stripe.py:253-293): data [nproj, nz, ni]
float32 -> ring-corrected copy.  ``StripeFW`` is the reusable operator for a
fixed chunk shape, working in place on padded sinograms
[nz, nproj + nproj//8, ni] (the layout the fused pipeline produces).
The wavelet filters come from :mod:`.wavelets`.
"""
from __future__ import annotations

import ctypes as C
import functools

import numpy as np
import torch

from .. import _lib
from .._handle import NativeHandle
from . import wavelets
from .proc_functions import prep_rows


class StripeFW(NativeHandle):
    _destroy = "tcb_stripe_fw_destroy"

    def __init__(self, nproj, nz, ni, sigma=1.0, wname="sym16", level=7):
        dl, dh, rl, rh = (np.ascontiguousarray(a, dtype=np.float64)
                          for a in wavelets.filter_bank(wname))
        P = C.POINTER(C.c_double)
        self._set(_lib.create("tcb_stripe_fw_create", int(nproj), int(nz), int(ni), int(level),
                              float(sigma), dl.ctypes.data_as(P), dh.ctypes.data_as(P),
                              rl.ctypes.data_as(P), rh.ctypes.data_as(P), len(rl)))
        self.nproj, self.nz, self.ni, self.level = int(nproj), int(nz), int(ni), int(level)
        self.nproj_pad = self.nproj + self.nproj // 8
        self.poff = (self.nproj_pad - self.nproj) // 2

    def apply_sino(self, sino, stream=None):
        """In place on sino [nz, nproj_pad, ni] float32 (pad rows zero on entry)."""
        assert sino.dtype == torch.float32 and sino.stride(2) == 1 and sino.stride(1) == self.ni
        _lib.call("tcb_stripe_fw_apply_sino", self._live(), sino.data_ptr(), sino.stride(0),
                  _lib.stream_ptr(stream))
        return sino


@functools.lru_cache(maxsize=8)
def _operator(nproj, nz, ni, sigma, wname, level, device_index):
    return StripeFW(nproj, nz, ni, sigma, wname, level)


def remove_stripe_fw(data, sigma, wname, level):
    """Remove stripes with wavelet filtering: data [nproj, nz, ni] -> new tensor."""
    nproj, nz, ni = data.shape
    op = _operator(nproj, nz, ni, float(sigma), str(wname), int(level),
                   data.device.index or 0)
    sino = torch.zeros((nz, op.nproj_pad, ni), dtype=torch.float32, device=data.device)
    src = data if data.dtype == torch.float32 else data.to(torch.float32)
    # [nproj, nz, ni] -> rows poff.. of [nz, nproj_pad, ni]
    prep_rows(sino, src, darkflat=False, minus_log=False, out_zstride=op.nproj_pad * ni,
              out_pstride=ni, out_poff=op.poff)
    op.apply_sino(sino)
    out = torch.empty((nproj, nz, ni), dtype=data.dtype, device=data.device)
    out.copy_(sino[:, op.poff:op.poff + nproj].permute(1, 0, 2))
    return out


# --------------------------------------------------------------------------
# Titarenko ring removal (remove_stripe.py:296-307)
# --------------------------------------------------------------------------
def ti_mask(n: int, mask_size: float) -> tuple[int, int]:
    """Column range [m0, m1) of the reference's
    mask[:, n//2 - ms//2 : n//2 + ms//2], ms = mask_size * n (Python slice
    rules; the reference only runs with an integer mask_size, since NumPy and
    CuPy reject float slice bounds)."""
    a, b = C.c_longlong(), C.c_longlong()
    _lib.call("tcb_stripe_ti_mask", int(n), float(mask_size), C.byref(a), C.byref(b))
    return a.value, b.value


class StripeTI(NativeHandle):
    """Titarenko ring removal for a fixed chunk shape, in place on sinograms
    [nz, nproj, ni] (any slice / angle strides with contiguous rows)."""
    _destroy = "tcb_stripe_ti_destroy"

    def __init__(self, nproj, nz, ni, beta=0.022, mask_size=1):
        self._set(_lib.create("tcb_stripe_ti_create", int(nproj), int(nz), int(ni), float(beta),
                              float(mask_size)))
        self.nproj, self.nz, self.ni = int(nproj), int(nz), int(ni)
        # the pipeline's stripe-operator interface (no angle padding)
        self.nproj_pad, self.poff = self.nproj, 0

    def apply_sino(self, sino, stream=None):
        """In place on sino [nz, >= nproj, ni] float32, angle rows 0..nproj-1."""
        assert sino.dtype == torch.float32 and sino.stride(2) == 1 and sino.shape[0] == self.nz
        _lib.call("tcb_stripe_ti_apply_sino", self._live(), sino.data_ptr(), sino.stride(0),
                  sino.stride(1), _lib.stream_ptr(stream))
        return sino


@functools.lru_cache(maxsize=8)
def _ti_operator(nproj, nz, ni, beta, mask_size, device_index):
    return StripeTI(nproj, nz, ni, beta, mask_size)


def remove_stripe_ti(data, beta, mask_size):
    """Remove stripes with Titarenko's method: data [nproj, nz, ni] float32 on
    the device, corrected in place and returned (like the reference)."""
    nproj, nz, ni = data.shape
    if data.dtype != torch.float32:
        raise ValueError("remove_stripe_ti: float32 data")
    op = _ti_operator(nproj, nz, ni, float(beta), float(mask_size), data.device.index or 0)
    op.apply_sino(data.permute(1, 0, 2))   # [nz, nproj, ni] view: strides (ni, nz*ni, 1)
    return data


# --------------------------------------------------------------------------
# Vo's all-stripe removal (remove_stripe.py:311-498)
# --------------------------------------------------------------------------
class StripeVO(NativeHandle):
    """remove_all_stripe for a fixed chunk shape, in place on sinograms
    [nz, nproj, ni] (any slice / angle strides with contiguous rows)."""
    _destroy = "tcb_stripe_vo_destroy"

    def __init__(self, nproj, nz, ni, snr=3.0, la_size=61, sm_size=21, dim=1):
        self._set(_lib.create("tcb_stripe_vo_create", int(nproj), int(nz), int(ni), float(snr),
                              int(la_size), int(sm_size), int(dim)))
        self.nproj, self.nz, self.ni = int(nproj), int(nz), int(ni)
        # the pipeline's stripe-operator interface (no angle padding)
        self.nproj_pad, self.poff = self.nproj, 0

    def apply_sino(self, sino, stream=None):
        """In place on sino [nz, >= nproj, ni] float32, angle rows 0..nproj-1."""
        assert sino.dtype == torch.float32 and sino.stride(2) == 1 and sino.shape[0] == self.nz
        _lib.call("tcb_stripe_vo_apply", self._live(), sino.data_ptr(), sino.stride(1),
                  sino.stride(0), _lib.stream_ptr(stream))
        return sino


@functools.lru_cache(maxsize=8)
def _vo_operator(nproj, nz, ni, snr, la_size, sm_size, dim, device_index):
    return StripeVO(nproj, nz, ni, snr, la_size, sm_size, dim)


def remove_all_stripe(tomo, snr=3, la_size=61, sm_size=21, dim=1):
    """Remove all types of stripe artifacts (Vo's method): tomo [nproj, nz, ni]
    float32 on the device, corrected in place and returned."""
    nproj, nz, ni = tomo.shape
    if tomo.dtype != torch.float32:
        raise ValueError("remove_all_stripe: float32 data")
    op = _vo_operator(nproj, nz, ni, float(snr), int(la_size), int(sm_size), int(dim),
                      tomo.device.index or 0)
    op.apply_sino(tomo.permute(1, 0, 2))   # [nz, nproj, ni] view
    return tomo
