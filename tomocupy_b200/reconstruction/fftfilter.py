"""Fused fp32 FBP filter (tcb_fftfilter_*).

The reference filters each sinogram row by edge-padding it to ``ne = 4n``,
multiplying its spectrum by ``w = wfilter * exp(-2*pi*i*(-center + sht + n/2)*t)``
and cropping ``n`` samples (src/tomocupy/reconstruction/backproj_functions.py:93-109
with cfunc_filter, src/cuda/cfunc_filter.cu:49-61).  That linear map is a
circular convolution of length ``L >= 2n`` with the impulse response
``hz = C2R(w)`` plus the folded padding columns; the native kernel runs it as
two shared-memory FFTs of length ``L`` per pair of rows, and can append
FourierRec's projection FFT so the gridding reads its output directly.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib
from .tcfilter import impulse_responses

MODES = {"rows": _lib.FFF_OUT_ROWS, "pairs": _lib.FFF_OUT_PAIRS,
         "spectrum": _lib.FFF_OUT_SPECTRUM}


def supported(n: int) -> bool:
    """Widths the fused filter handles (convolution length <= 8192)."""
    return 2 <= int(n) <= 4096


def spectrum_supported(n: int) -> bool:
    """Widths for which the projection FFT can be fused (power of two >= 256)."""
    n = int(n)
    return 256 <= n <= 4096 and n & (n - 1) == 0


def operator_columns(hz: np.ndarray, n: int, pad: int):
    """float64 (h_L, A, B): the circular-convolution kernel and the padding columns.

    Host-side statement of what tcb_fftfilter_set_kernels builds (used by
    the tests): ``y = ifft(fft(x_L) * fft(h_L))[:n] + x[0] * A + x[n-1] * B``.
    """
    ne = hz.shape[0]
    L = 256
    while L < 2 * n:
        L *= 2
    hL = np.zeros(L)
    hL[:n] = hz[:n]
    hL[L - n + 1:] = hz[ne - n + 1:]
    ext = np.concatenate([hz, hz])
    cs = np.concatenate([[0.0], np.cumsum(ext)])
    j = np.arange(n)
    col0 = cs[j + pad + 1 + ne] - cs[j + ne]
    coln = cs[j - n + 2 + ne] - cs[j + pad - ne + 1 + ne]
    A = col0 - hz[j % ne]
    B = coln - hz[(j - n + 1) % ne]
    return hL, A, B


class FFTFilter:
    """Fused filter for [nz, nproj, n] fp32 sinogram rows."""

    def __init__(self, n: int, nproj: int, nz: int, nkern: int = 1, device=None):
        self.n, self.nproj, self.nz, self.nkern = int(n), int(nproj), int(nz), int(nkern)
        self.device = torch.device(device or "cuda")
        with torch.cuda.device(self.device):
            self.handle = _lib.create("tcb_fftfilter_create", self.nproj, self.nz, self.n,
                                      self.nkern)
        self.ne = None

    def set_kernels(self, wfilter: np.ndarray, ne: int, center: float, sht=0.0) -> None:
        """One kernel, or ``nkern`` kernels for the centre shifts ``sht``."""
        sht = np.atleast_1d(np.asarray(sht, dtype=np.float64))
        if sht.size == 1 and self.nkern > 1:
            sht = np.repeat(sht, self.nkern)
        if sht.size != self.nkern:
            raise ValueError(f"need {self.nkern} centre shifts, got {sht.size}")
        hz = np.ascontiguousarray(impulse_responses(wfilter, ne, self.n, center, sht))
        pad = ne // 2 - self.n // 2
        with torch.cuda.device(self.device):
            _lib.call("tcb_fftfilter_set_kernels", self.handle,
                      hz.ctypes.data_as(C.c_void_p), ne, pad,
                      torch.cuda.current_stream(self.device).cuda_stream)
        self.ne = ne

    def apply(self, x: torch.Tensor, out: torch.Tensor, mode: str = "rows", *, kern0: int = 0,
              xoff: int = 0, stream=None) -> torch.Tensor:
        """Filter rows x [nz, nproj, ldx] (columns [xoff, xoff + n)) into ``out``.

        ``rows``: out float32 [nz, nproj, ldo].  ``pairs``: out complex64
        [nz/2, nproj, n], slice z real part, slice z + nz/2 imaginary part.
        ``spectrum``: the same packed rows after a forward FFT of length n.
        """
        nz = x.shape[0]
        assert x.dtype == torch.float32 and x.stride(2) == 1
        assert x.shape[1] == self.nproj and x.stride(0) == self.nproj * x.stride(1)
        assert x.shape[2] >= xoff + self.n
        m = MODES[mode]
        if mode == "rows":
            assert out.dtype == torch.float32 and out.stride(2) == 1
            assert out.shape[0] >= nz and out.shape[1] == self.nproj
            assert out.shape[2] >= self.n and out.stride(0) == self.nproj * out.stride(1)
            ldo = out.stride(1)
        else:
            assert out.dtype == torch.complex64 and out.is_contiguous()
            assert tuple(out.shape) == (nz // 2, self.nproj, self.n)
            ldo = self.n
        _lib.call("tcb_fftfilter_apply", self.handle, _lib.ptr(x), x.stride(1), int(xoff), nz,
                  int(kern0), _lib.ptr(out), m, ldo, _lib.stream_ptr(stream))
        return out

    def free(self) -> None:
        if self.handle:
            _lib.call("tcb_fftfilter_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
