"""Drop-in for the reference module ``tomocupy.cfunc_linerec``.

Same constructor and methods as the SWIG class (src/cuda/cfunc_linerec.i:9-25);
every method accumulates into ``f``.
"""
from __future__ import annotations

from . import _lib


class cfunc_linerec:
    _precision = _lib.TCB_FLOAT32

    def __init__(self, nproj, nz, n, ncproj, ncz):
        self._h = _lib.create("tcb_linerec_create", int(nproj), int(nz), int(n), int(ncproj),
                              int(ncz), self._precision)
        self._dims = dict(n=int(n), nproj=int(nproj), nz=int(nz), ncproj=int(ncproj),
                          ncz=int(ncz))

    n = property(lambda self: self._dims["n"])
    nproj = property(lambda self: self._dims["nproj"])
    nz = property(lambda self: self._dims["nz"])
    ncproj = property(lambda self: self._dims["ncproj"])
    ncz = property(lambda self: self._dims["ncz"])

    def _live(self):
        if self._h is None:
            raise _lib.TcbError(6, "cfunc_linerec", "object was freed")
        return self._h

    def backprojection(self, f_, g_, theta, phi, sz, stream_):
        _lib.call("tcb_linerec_backprojection", self._live(), _lib.ptr(f_), _lib.ptr(g_),
                  _lib.ptr(theta), float(phi), int(sz), _lib.stream_ptr(stream_))

    def backprojection_try(self, f_, g_, theta_, sh_, phi, sz, stream_):
        _lib.call("tcb_linerec_backprojection_try", self._live(), _lib.ptr(f_), _lib.ptr(g_),
                  _lib.ptr(theta_), _lib.ptr(sh_), float(phi), int(sz),
                  _lib.stream_ptr(stream_))

    def backprojection_try_lamino(self, f_, g_, theta_, phi_, sz, stream_):
        _lib.call("tcb_linerec_backprojection_try_lamino", self._live(), _lib.ptr(f_),
                  _lib.ptr(g_), _lib.ptr(theta_), _lib.ptr(phi_), int(sz),
                  _lib.stream_ptr(stream_))

    def timed_out(self) -> bool:
        """True when a TMA wait of the float32 backprojection gave up (synchronises;
        not in the reference)."""
        import ctypes as C
        v = C.c_int(0)
        _lib.call("tcb_linerec_status", self._live(), C.byref(v))
        return bool(v.value)

    def free(self):
        if getattr(self, "_h", None) is not None:
            _lib.call("tcb_linerec_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
