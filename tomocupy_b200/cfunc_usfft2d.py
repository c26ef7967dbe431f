"""Drop-in for ``tomocupy.cfunc_usfft2d`` (src/cuda/cfunc_usfft2d.i:9-18):
``fwd`` and ``adj`` with the reference's argument order (the reconstruction
path, LamFourierRec.usfft2d_adj, uses the adjoint)."""
from __future__ import annotations

from . import _lib
from ._handle import NativeHandle


class cfunc_usfft2d(NativeHandle):
    _destroy = "tcb_usfft2d_destroy"

    def __init__(self, n0, n1, n2, ntheta, detw, deth):
        self._set(_lib.create("tcb_usfft2d_create", int(n0), int(n1), int(n2), int(ntheta),
                              int(detw), int(deth)))

    def adj(self, f_, g_, theta_, phi, k, deth0, stream_):
        _lib.call("tcb_usfft2d_adj", self._live(), _lib.ptr(f_), _lib.ptr(g_), _lib.ptr(theta_),
                  float(phi), int(k), int(deth0), _lib.stream_ptr(stream_))

    def adj_rows(self, S2, S1, theta, phi, row0, nrows, deth_full, stream_):
        """Fused adjoint on rows [row0, row0+nrows) of the whole stage-1 spectrum."""
        _lib.call("tcb_usfft2d_adj_rows", self._live(), _lib.ptr(S2), _lib.ptr(S1),
                  _lib.ptr(theta), float(phi), int(row0), int(nrows), int(deth_full),
                  _lib.stream_ptr(stream_))

    def set_storage(self, precision: int, in_scale=None, out_inv_scale=None) -> None:
        """Not in the reference: _lib.TCB_FLOAT16 stores the stage arrays in complex
        fp16, with optional per-angle / per-row power-of-two scale arrays."""
        _lib.call("tcb_usfft2d_set_storage", self._live(), int(precision), _lib.ptr(in_scale), _lib.ptr(out_inv_scale))

    def sample_positions(self, x, y, theta_, phi, k, deth0, stream_):
        """x, y fp32 [ntheta, deth, detw] <- the sample positions take_x computes
        for chunk k, as the gridding kernel computes them (a test hook; not in
        the reference)."""
        _lib.call("tcb_usfft2d_sample_positions", self._live(), _lib.ptr(x), _lib.ptr(y),
                  _lib.ptr(theta_), float(phi), int(k), int(deth0), _lib.stream_ptr(stream_))

    def fwd(self, g_, f_, theta_, phi, k, deth0, stream_):
        """g [2*ntheta, deth, detw/2+1] complex <- f [n1, n2 slabs, n0] complex."""
        _lib.call("tcb_usfft2d_fwd", self._live(), _lib.ptr(g_), _lib.ptr(f_), _lib.ptr(theta_),
                  float(phi), int(k), int(deth0), _lib.stream_ptr(stream_))
