"""Mixed-precision FBP filter on the tensor cores (tcb_tcfilter_*).

The reference filters each sinogram row by edge-padding it to ``ne``,
multiplying its spectrum by ``w = wfilter * exp(-2*pi*i*(-center + sht + n/2)*t)``
and cropping ``n`` samples (src/tomocupy/reconstruction/backproj_functions.py:93-109
with cfunc_filter, src/cuda/cfunc_filter.cu:49-61).  The chain is linear in
the row, so it is an ``n x n`` matrix ``T`` per filter kernel; the native
code builds ``T`` in float64 from the impulse response ``hz = C2R(w)``
computed here in float64 (spectrum and phase ramp included), and applies it
as an fp16 tcgen05 GEMM with a hi/lo split-precision correction and fp32
accumulation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib


def impulse_responses(wfilter: np.ndarray, ne: int, n: int, center: float,
                      sht) -> np.ndarray:
    """float64 [nk, ne]: unnormalised C2R of ``wfilter * exp(-2 pi i (-center + sht + n/2) t)``.

    ``wfilter`` is the reference's float32 spectrum (``ne/2 + 1`` values, the
    ``1/ne`` of the inverse FFT folded in); ``t = k/ne``.  A C2R, like the
    reference's cuFFT C2R, ignores the imaginary parts of the DC and Nyquist
    bins.
    """
    wf = np.asarray(wfilter, dtype=np.float64)
    assert wf.shape == (ne // 2 + 1,)
    sht = np.atleast_1d(np.asarray(sht, dtype=np.float64))
    t = np.arange(ne // 2 + 1, dtype=np.float64) / ne
    shift = -float(center) + sht + n / 2
    w = wf[None, :] * np.exp(-2j * np.pi * shift[:, None] * t[None, :])
    return np.fft.irfft(w, ne, axis=1) * ne


def toeplitz_operator(hz: np.ndarray, n: int, pad: int) -> np.ndarray:
    """float64 [n, n] matrix of edge-pad -> circular convolution with hz -> crop.

    ``T[j, i] = hz[(j - i) mod ne]`` with the left padding folded into column 0
    and the right padding into column ``n - 1``; host-side statement of what
    tcb_tcfilter_set_kernels builds on the device.
    """
    ne = hz.shape[0]
    j = np.arange(n)[:, None]
    i = np.arange(n)[None, :]
    T = hz[(j - i) % ne].copy()
    ext = np.concatenate([hz, hz])  # ext[d + ne] = hz[d mod ne] for d in [-ne, ne)
    cs = np.concatenate([[0.0], np.cumsum(ext)])
    jj = np.arange(n)
    T[:, 0] = cs[jj + pad + 1 + ne] - cs[jj + ne]
    T[:, n - 1] = cs[jj - n + 2 + ne] - cs[jj + pad - ne + 1 + ne]
    return T


class TCFilter:
    """Tensor-core filter for [nz, nproj, n] sinogram rows given as fp16 hi/lo planes."""

    def __init__(self, n: int, nproj: int, nz: int, nkern: int = 1, device=None):
        self.n, self.nproj, self.nz, self.nkern = int(n), int(nproj), int(nz), int(nkern)
        self.device = torch.device(device or "cuda")
        with torch.cuda.device(self.device):
            self.handle = _lib.create("tcb_tcfilter_create", self.nproj, self.nz, self.n,
                                      self.nkern)
        self.ne = None

    def set_kernels(self, wfilter: np.ndarray, ne: int, center: float, sht=0.0) -> None:
        """Build the operator(s): one kernel, or ``nkern`` kernels for shifts ``sht``."""
        sht = np.atleast_1d(np.asarray(sht, dtype=np.float64))
        if sht.size == 1 and self.nkern > 1:
            sht = np.repeat(sht, self.nkern)
        if sht.size != self.nkern:
            raise ValueError(f"need {self.nkern} centre shifts, got {sht.size}")
        hz = np.ascontiguousarray(impulse_responses(wfilter, ne, self.n, center, sht))
        pad = ne // 2 - self.n // 2
        with torch.cuda.device(self.device):
            _lib.call("tcb_tcfilter_set_kernels", self.handle,
                      hz.ctypes.data_as(C.c_void_p), ne, pad,
                      torch.cuda.current_stream(self.device).cuda_stream)
        self.ne = ne

    def apply(self, x_hi: torch.Tensor, x_lo: torch.Tensor, out: torch.Tensor, *,
              pairs: bool = False, kern0: int = 0, stream=None) -> torch.Tensor:
        """Filter [nz, nproj, lda] hi/lo planes into ``out``.

        ``pairs=False``: out float32 [nz, nproj, ldo].  ``pairs=True``: out
        complex64 [nz/2, nproj, n] in the packed layout of FourierRec (slice z
        real part, slice z + nz/2 imaginary part).
        """
        nz = x_hi.shape[0]
        assert x_hi.shape == x_lo.shape and x_hi.dtype == torch.float16
        assert x_lo.dtype == torch.float16
        assert x_hi.shape[1] == self.nproj and x_hi.stride(2) == 1
        assert x_hi.stride(0) == self.nproj * x_hi.stride(1) and x_lo.stride() == x_hi.stride()
        lda = x_hi.stride(1)
        if pairs:
            assert out.dtype == torch.complex64 and out.is_contiguous()
            assert tuple(out.shape) == (nz // 2, self.nproj, self.n)
            mode, ldo = _lib.TCF_OUT_PAIRS, self.n
        else:
            assert out.dtype == torch.float32 and out.stride(2) == 1
            assert out.shape[0] >= nz and out.shape[1] == self.nproj and out.shape[2] >= self.n
            assert out.stride(0) == self.nproj * out.stride(1)
            mode, ldo = _lib.TCF_OUT_ROWS, out.stride(1)
        _lib.call("tcb_tcfilter_apply", self.handle, _lib.ptr(x_hi), _lib.ptr(x_lo), lda, nz,
                  int(kern0), _lib.ptr(out), mode, ldo, _lib.stream_ptr(stream))
        return out

    def timed_out(self) -> bool:
        """True when a kernel of this handle gave up on a bounded wait (synchronises)."""
        v = C.c_int(0)
        _lib.call("tcb_tcfilter_status", self.handle, C.byref(v))
        return bool(v.value)

    def free(self) -> None:
        if self.handle:
            _lib.call("tcb_tcfilter_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def split16(x: torch.Tensor):
    """(hi, lo) fp16 planes with hi = fp16(x), lo = fp16(x - hi)."""
    hi = x.to(torch.float16)
    lo = (x - hi.to(torch.float32)).to(torch.float16)
    return hi, lo
