"""Drop-in for the reference module ``tomocupy.cfunc_filter``.

Same constructor and ``filter(g, w, stream)`` as the SWIG class
(src/cuda/cfunc_filter.i:9-21): ``g`` real [nz, nproj, n] filtered in place,
``w`` complex [nz, n/2+1].
"""
from __future__ import annotations

from . import _lib


class cfunc_filter:
    _precision = _lib.TCB_FLOAT32

    def __init__(self, nproj, nz, n):
        self._h = _lib.create("tcb_filter_create", int(nproj), int(nz), int(n),
                              self._precision)
        self._n, self._nproj, self._nz = int(n), int(nproj), int(nz)

    n = property(lambda self: self._n)
    nproj = property(lambda self: self._nproj)
    nz = property(lambda self: self._nz)

    def filter(self, g, w, stream):
        if self._h is None:
            raise _lib.TcbError(6, "cfunc_filter.filter", "object was freed")
        _lib.call("tcb_filter_apply", self._h, _lib.ptr(g), _lib.ptr(w), _lib.stream_ptr(stream))

    def free(self):
        if getattr(self, "_h", None) is not None:
            _lib.call("tcb_filter_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
