"""FBP filter: spectrum construction and application.

``FBPFilter`` mirrors the reference class (src/tomocupy/reconstruction/fbp_filter.py:45-118):
``calc_filter`` builds the quadrature-corrected window in float64 (NumPy stands
in for CuPy; the operation order is kept so the float32 result matches), and
``filter`` applies per-slice spectra through the native ``cfunc_filter``.
"""
from __future__ import annotations

import functools

import numpy as np

from .. import cfunc_filter, cfunc_filterfp16

FILTERS = ("none", "ramp", "shepp", "cosine", "cosine2", "hamming", "hann", "parzen")


def _wint(n: int, t: np.ndarray) -> np.ndarray:
    """Quadrature weights of the ramp |t| (fbp_filter.py:91-118), float64."""
    N = len(t)
    s = np.linspace(1e-40, 1, n)
    # inverse Vandermonde matrix
    tmp1 = np.arange(n)
    tmp2 = np.arange(1, n + 2)
    iv = np.linalg.inv(np.exp(np.outer(tmp1, np.log(s))))
    # integration over short intervals
    u = np.diff(np.exp(np.outer(tmp2, np.log(s))) * np.tile(1.0 / tmp2[..., np.newaxis], [1, n]))
    W1 = np.matmul(iv, u[1:n + 1, :])  # x*pn(x) term
    W2 = np.matmul(iv, u[0:n, :])  # const*pn(x) term
    # compensate for overlapping short intervals
    tmp1 = np.arange(1, n)
    tmp2 = (n - 1) * np.ones((N - 2 * (n - 1) - 1))
    tmp3 = np.arange(n - 1, 0, -1)
    p = 1 / np.concatenate((tmp1, tmp2, tmp3))
    w = np.zeros(N)
    for j in range(N - n + 1):
        # change of coordinates, constant and linear parts
        W = ((t[j + n - 1] - t[j]) ** 2) * W1 + (t[j + n - 1] - t[j]) * t[j] * W2
        for k in range(n - 1):
            w[j:j + n] = w[j:j + n] + p[j + k] * W[:, k]
    wn = w
    wn[-40:] = (w[-40]) / (N - 40) * np.arange(N - 40, N)
    return wn


@functools.lru_cache(maxsize=16)
def _calc_filter_cached(ne: int, name: str) -> np.ndarray:
    d = 0.5
    t = np.arange(0, ne / 2 + 1) / ne
    if name == "none":
        wfa = ne * 0.5 + t * 0
        wfa[0] *= 2  # fixed later
    elif name == "ramp":
        wfa = ne * 0.5 * _wint(12, t)
    elif name == "shepp":
        wfa = ne * 0.5 * _wint(12, t) * np.sinc(t / (2 * d)) * (t / d <= 2)
    elif name == "cosine":
        wfa = ne * 0.5 * _wint(12, t) * np.cos(np.pi * t / (2 * d)) * (t / d <= 1)
    elif name == "cosine2":
        wfa = ne * 0.5 * _wint(12, t) * (np.cos(np.pi * t / (2 * d))) ** 2 * (t / d <= 1)
    elif name == "hamming":
        wfa = ne * 0.5 * _wint(12, t) * (.54 + .46 * np.cos(np.pi * t / d)) * (t / d <= 1)
    elif name == "hann":
        wfa = ne * 0.5 * _wint(12, t) * (1 + np.cos(np.pi * t / d)) / 2.0 * (t / d <= 1)
    elif name == "parzen":
        wfa = ne * 0.5 * _wint(12, t) * pow(1 - t / d, 3) * (t / d <= 1)
    else:
        raise ValueError(f"unknown FBP filter {name!r}; choices: {FILTERS}")
    wfa = 2 * wfa * (wfa >= 0)
    wfa[0] *= 2
    # the inverse-FFT normalisation 1/ne is folded in here
    wfa = wfa.astype("float32") / ne
    wfa.setflags(write=False)
    return wfa


def calc_filter(ne: int, name: str) -> np.ndarray:
    """float32 [ne/2+1] filter spectrum (a fresh, writable copy)."""
    return _calc_filter_cached(int(ne), str(name)).copy()


class FBPFilter:
    """Same constructor and methods as the reference ``FBPFilter``."""

    def __init__(self, n, ntheta, nz, dtype):
        mod = cfunc_filterfp16 if dtype == "float16" else cfunc_filter
        self.fslv = mod.cfunc_filter(ntheta, nz, n)
        self.n = n
        self.dtype = dtype

    def filter(self, data, w, stream):
        """data real [nz, ntheta, n] filtered in place with w complex64 [nz, n/2+1]."""
        import torch
        data = data.contiguous()
        w = torch.view_as_real(w.contiguous()).to(data.dtype).contiguous()
        self.fslv.filter(data, w, stream)
        return data

    def calc_filter(self, filter):
        return calc_filter(self.n, filter)
