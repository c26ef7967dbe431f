"""Orthogonal wavelet filter banks for the Fourier-wavelet ring removal.

The reference takes its filters from PyWavelets (``pywt.Wavelet(name)``,
src/tomocupy/processing/remove_stripe.py:158-184), which is not available
here.  The filters are derived instead with Daubechies' published
construction (I. Daubechies, "Ten Lectures on Wavelets", 1992, ch. 6 and
8.1): the scaling filter with N vanishing moments is
H(z) = sqrt(2) ((1+z^-1)/2)^N Q(z), where |Q|^2 = P(sin^2(w/2)) with
P(y) = sum_{k<N} C(N-1+k, k) y^k.  Each root y_k of P gives the reciprocal
pair z + 1/z = 2 - 4 y_k; keeping the roots inside the unit circle gives the
minimum-phase (extremal phase) filters "dbN"; choosing, per conjugate root
group, the member that makes the phase closest to linear gives the least
asymmetric filters "symN".

Filter-bank conventions (PyWavelets' ``filter_bank``): rec_lo is the scaling
filter (sum sqrt(2)), dec_lo = rec_lo reversed, dec_hi[k] = (-1)^(k+1)
rec_lo[k], rec_hi = dec_hi reversed.
"""
from __future__ import annotations

import functools
import itertools
from math import comb

import numpy as np

SUPPORTED = ("haar", "db1", "db5", "sym5", "sym16")


def _p_roots(N: int) -> np.ndarray:
    """Roots of P(y) = sum_{k<N} C(N-1+k, k) y^k, polished by Newton steps."""
    coeffs = [comb(N - 1 + k, k) for k in range(N)]  # ascending powers
    if N == 1:
        return np.zeros(0, dtype=complex)
    r = np.roots(coeffs[::-1]).astype(complex)
    c = np.array(coeffs, dtype=float)
    dc = np.array([k * c[k] for k in range(1, N)], dtype=float)
    for _ in range(8):
        p = np.polyval(c[::-1], r)
        dp = np.polyval(dc[::-1], r)
        r = r - p / dp
    return r


def _z_pair(y: complex):
    """Both z with z + 1/z = 2 - 4y (inside first)."""
    b = 2 - 4 * y
    s = np.sqrt(b * b - 4 + 0j)
    z1, z2 = (b + s) / 2, (b - s) / 2
    return (z1, z2) if abs(z1) <= abs(z2) else (z2, z1)


def _filter_from_roots(N: int, zs) -> np.ndarray:
    """Real scaling filter from (1+z)^N times prod (z - z_k), normalised to sum sqrt(2)."""
    poly = np.array([comb(N, k) for k in range(N + 1)], dtype=complex)
    for z in zs:
        poly = np.convolve(poly, np.array([1.0, -z]))
    h = poly.real
    return h * (np.sqrt(2.0) / h.sum())


def _root_groups(N: int):
    """Per conjugate group of P-roots: the two candidate z-root sets (inside, outside)."""
    ys = _p_roots(N)
    groups, used = [], np.zeros(len(ys), bool)
    for i, y in enumerate(ys):
        if used[i]:
            continue
        used[i] = True
        zin, zout = _z_pair(y)
        if abs(y.imag) < 1e-9:
            groups.append(([zin.real + 0j], [zout.real + 0j]))
        else:
            j = int(np.argmin(np.abs(ys - np.conj(y)) + used * 1e9))
            used[j] = True
            groups.append(([zin, np.conj(zin)], [zout, np.conj(zout)]))
    return groups


def _phase_nonlinearity(h: np.ndarray) -> float:
    w = np.linspace(0, np.pi, 1025)[1:-1]
    H = np.polyval(h[::-1], np.exp(-1j * w))  # sum h_k e^{-i w k}
    ph = np.unwrap(np.angle(H))
    A = np.vstack([w, np.ones_like(w)]).T
    coef, res, *_ = np.linalg.lstsq(A, ph, rcond=None)
    return float(np.sum((A @ coef - ph) ** 2))


@functools.lru_cache(maxsize=None)
def scaling_filter(name: str) -> tuple:
    """rec_lo of the wavelet (float64 tuple)."""
    if name in ("haar", "db1", "sym1"):
        return (np.sqrt(0.5), np.sqrt(0.5))
    fam, N = name[:-len(name.lstrip("dbsym"))] if False else None, None
    if name.startswith("db"):
        N = int(name[2:])
        zs = [z for g in _root_groups(N) for z in g[0]]
        h = _filter_from_roots(N, zs)
        # minimum phase: energy at the start
        if np.sum(h[:len(h) // 2] ** 2) < np.sum(h[len(h) // 2:] ** 2):
            h = h[::-1]
        return tuple(h)
    if name.startswith("sym"):
        N = int(name[3:])
        groups = _root_groups(N)
        best, best_h = None, None
        for choice in itertools.product((0, 1), repeat=len(groups)):
            zs = [z for g, c in zip(groups, choice) for z in g[c]]
            h = _filter_from_roots(N, zs)
            q = _phase_nonlinearity(h)
            if best is None or q < best - 1e-12:
                best, best_h = q, h
        h = best_h
        # of the two mirror images, keep the one whose energy centroid lies
        # at or after the filter centre
        k = np.arange(len(h))
        if np.sum(k * h ** 2) < (len(h) - 1) / 2 * np.sum(h ** 2):
            h = h[::-1]
        return tuple(h)
    raise ValueError(f"unsupported wavelet {name!r}; choices: {SUPPORTED}")


def filter_bank(name: str):
    """(dec_lo, dec_hi, rec_lo, rec_hi) as float64 arrays."""
    rec_lo = np.array(scaling_filter(name))
    dec_lo = rec_lo[::-1].copy()
    k = np.arange(len(rec_lo))
    dec_hi = ((-1.0) ** (k + 1)) * rec_lo
    rec_hi = dec_hi[::-1].copy()
    return dec_lo, dec_hi, rec_lo, rec_hi


def dwt_coeff_len(n: int, L: int) -> int:
    """Output length of one DWT level in 'symmetric' mode: floor((n + L - 1) / 2)."""
    return (n + L - 1) // 2
