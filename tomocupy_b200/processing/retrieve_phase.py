"""Single-distance phase retrieval of projections (Paganin, generalised
Paganin, Farago).

Mirrors ``paganin_filter`` and ``farago_filter``
(src/tomocupy/processing/retrieve_phase.py:57-145): same names, argument
order, units (pixel_size and dist in cm, energy in keV, W in cm) and in-place
semantics on ``data`` [nproj, dy, dz] float32, which is also returned.  The
work runs in ``tcb_phase_apply``: edge padding, an R2C 2D transform, the
even part of the normalised filter, a C2R 2D transform and the crop (equal
to the reference's real(ifft2(fft2(prj) * filter)) because the filter is
real).  Handles are cached per geometry and parameter set, so a chunked
driver builds each filter once (the reference rebuilds it per call).
"""
from __future__ import annotations

import ctypes as C

import torch

from .. import _lib

__all__ = ["paganin_filter", "farago_filter", "PhaseFilter", "pads"]

METHODS = {"paganin": _lib.TCB_PHASE_PAGANIN, "Gpaganin": _lib.TCB_PHASE_GPAGANIN,
           "farago": _lib.TCB_PHASE_FARAGO}

# padded images per transform batch are capped at this many bytes (input
# image, its spectrum and the filter share the budget)
BATCH_BYTES = 1 << 30


def pads(dy: int, dz: int, pixel_size: float, dist: float, energy: float,
         pad: bool = True) -> tuple[int, int]:
    """Edge padding (rows, columns) on each side, as _calc_pad chooses it
    (retrieve_phase.py:178-226)."""
    py, pz = C.c_size_t(), C.c_size_t()
    _lib.call("tcb_phase_pads", int(dy), int(dz), float(pixel_size), float(dist), float(energy),
              int(bool(pad)), C.byref(py), C.byref(pz))
    return py.value, pz.value


class PhaseFilter:
    """A resident phase-retrieval operator for [*, dy, dz] projections."""

    def __init__(self, dy, dz, method="paganin", pixel_size=1e-4, dist=50, energy=20,
                 alpha=1e-3, db=1000, W=2e-4, pad=True, batch=None):
        if method not in METHODS:
            raise ValueError(f"unknown phase retrieval method {method!r}")
        self.dy, self.dz = int(dy), int(dz)
        py, pz = pads(dy, dz, pixel_size, dist, energy, pad)
        ny, nz = self.dy + 2 * py, self.dz + 2 * pz
        if batch is None:
            batch = max(1, min(64, BATCH_BYTES // (ny * nz * 8)))
        self.batch = int(batch)
        self._h = _lib.create("tcb_phase_create", self.batch, self.dy, self.dz, METHODS[method],
                              float(pixel_size), float(dist), float(energy), float(alpha),
                              float(db), float(W), int(bool(pad)))
        self.py, self.pz = py, pz

    def apply(self, data: torch.Tensor, stream=None) -> torch.Tensor:
        """In place on data [nproj, dy, dz] float32 (device, contiguous)."""
        if self._h is None:
            raise _lib.TcbError(6, "PhaseFilter", "object was freed")
        if (data.dtype != torch.float32 or data.dim() != 3 or not data.is_cuda
                or not data.is_contiguous() or tuple(data.shape[1:]) != (self.dy, self.dz)):
            raise ValueError(f"data must be a contiguous CUDA float32 [*, {self.dy}, {self.dz}] "
                             f"tensor, got {tuple(data.shape)} {data.dtype}")
        _lib.call("tcb_phase_apply", self._h, _lib.ptr(data), int(data.shape[0]),
                  _lib.stream_ptr(stream))
        return data

    def free(self) -> None:
        if self._h is not None:
            _lib.call("tcb_phase_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


_CACHE: dict[tuple, PhaseFilter] = {}


def _cached(dy, dz, method, pixel_size, dist, energy, alpha, db, W, pad) -> PhaseFilter:
    key = (torch.cuda.current_device(), dy, dz, method, pixel_size, dist, energy, alpha, db, W,
           bool(pad))
    op = _CACHE.get(key)
    if op is None:
        if len(_CACHE) >= 8:
            _CACHE.pop(next(iter(_CACHE))).free()
        op = _CACHE[key] = PhaseFilter(dy, dz, method, pixel_size, dist, energy, alpha, db, W,
                                       pad)
    return op


def paganin_filter(data, pixel_size=1e-4, dist=50, energy=20, alpha=1e-3, method="paganin",
                   db=1000, W=2e-4, pad=True):
    """Paganin ('paganin') or generalised Paganin ('Gpaganin') phase retrieval
    in place on projections [nproj, dy, dz] (retrieve_phase.py:57-99)."""
    if method not in ("paganin", "Gpaganin"):
        raise ValueError(f"paganin_filter: method {method!r}")
    _, dy, dz = data.shape
    return _cached(dy, dz, method, pixel_size, dist, energy, alpha, db, W, pad).apply(data)


def farago_filter(data, pixel_size=1e-4, dist=50, energy=20, db=1000, method="farago", pad=True):
    """Farago phase retrieval in place on projections [nproj, dy, dz]
    (retrieve_phase.py:101-127)."""
    if method != "farago":
        raise ValueError(f"farago_filter: method {method!r}")
    _, dy, dz = data.shape
    return _cached(dy, dz, method, pixel_size, dist, energy, 1e-3, db, 2e-4, pad).apply(data)
