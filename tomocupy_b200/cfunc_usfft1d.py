"""Drop-in for ``tomocupy.cfunc_usfft1d`` (src/cuda/cfunc_usfft1d.i:9-18):
``fwd`` and ``adj`` with the reference's argument order (the reconstruction
path, LamFourierRec.usfft1d_adj, uses the adjoint)."""
from __future__ import annotations

from . import _lib
from ._handle import NativeHandle


class cfunc_usfft1d(NativeHandle):
    _destroy = "tcb_usfft1d_destroy"

    def __init__(self, n0, n1, n2, deth):
        self._set(_lib.create("tcb_usfft1d_create", int(n0), int(n1), int(n2), int(deth)))

    def adj(self, f_, g_, phi, stream_):
        _lib.call("tcb_usfft1d_adj", self._live(), _lib.ptr(f_), _lib.ptr(g_), float(phi),
                  _lib.stream_ptr(stream_))

    def set_storage(self, precision: int, in_scale=None) -> None:
        """Not in the reference: _lib.TCB_FLOAT16 stores the stage arrays in complex
        fp16, with optional per-angle / per-row power-of-two scale arrays."""
        _lib.call("tcb_usfft1d_set_storage", self._live(), int(precision), _lib.ptr(in_scale))

    def fwd(self, g_, f_, phi, stream_):
        """g [n1, deth/2+1, n2] complex <- f [n1, n0 (height), n2] real."""
        _lib.call("tcb_usfft1d_fwd", self._live(), _lib.ptr(g_), _lib.ptr(f_), float(phi),
                  _lib.stream_ptr(stream_))
