"""Drop-in for ``tomocupy.cfunc_fft2d`` (src/cuda/cfunc_fft2d.i:9-18)."""
from __future__ import annotations

from . import _lib
from ._handle import NativeHandle


class cfunc_fft2d(NativeHandle):
    _destroy = "tcb_fft2d_destroy"

    def __init__(self, ntheta, detw, deth):
        self._set(_lib.create("tcb_fft2d_create", int(ntheta), int(detw), int(deth)))

    def fwd(self, g_, f_, stream_):
        """g complex [ntheta, deth, detw/2+1] <- 2D R2C of f [ntheta, deth, detw]."""
        _lib.call("tcb_fft2d_fwd", self._live(), _lib.ptr(g_), _lib.ptr(f_),
                  _lib.stream_ptr(stream_))

    def adj(self, g_, f_, stream_):
        """No-op, as in the reference (its body is commented out, cfunc_fft2d.cu:39-50)."""
        self._live()
