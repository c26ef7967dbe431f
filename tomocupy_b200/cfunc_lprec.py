"""Drop-in for ``tomocupy.cfunc_lprec`` (src/cuda/cfunc_lprec.i:11-29)."""
from __future__ import annotations

from . import _lib
from ._handle import NativeHandle


class cfunc_lprec(NativeHandle):
    _destroy = "tcb_lprec_destroy"
    _precision = _lib.TCB_FLOAT32

    def __init__(self, nproj, nz, n, ntheta, nrho):
        self._set(_lib.create("tcb_lprec_create", int(nproj), int(nz), int(n), int(ntheta),
                              int(nrho), self._precision))
        self.n, self.nproj, self.nz, self.ntheta, self.nrho = (int(n), int(nproj), int(nz),
                                                               int(ntheta), int(nrho))

    def setgrids(self, fz, lp2p1, lp2p2, lp2p1w, lp2p2w, C2lp1, C2lp2, lpids, wids, cids,
                 nlpids, nwids, ncids):
        """Borrow the device grids (the caller keeps them alive, as LpRec does)."""
        p = _lib.ptr
        _lib.call("tcb_lprec_setgrids", self._live(), p(fz), p(lp2p1), p(lp2p2), p(lp2p1w),
                  p(lp2p2w), p(C2lp1), p(C2lp2), p(lpids), p(wids), p(cids), int(nlpids),
                  int(nwids), int(ncids))

    def backprojection(self, f, g, stream):
        _lib.call("tcb_lprec_backprojection", self._live(), _lib.ptr(f), _lib.ptr(g),
                  _lib.stream_ptr(stream))
