"""``LamFourierRec`` (src/tomocupy/reconstruction/lamfourierrec.py:46-73) over the
native fft2d / usfft2d / usfft1d operators, same constructor and methods."""
from __future__ import annotations

from .. import cfunc_fft2d, cfunc_usfft1d, cfunc_usfft2d


class LamFourierRec:
    """Laminographic backprojection by the Fourier-based method."""

    def __init__(self, n0, n1, n2, ntheta, detw, deth, n1c, nthetac, dethc):
        self.n0, self.n1, self.n2 = n0, n1, n2
        self.ntheta, self.detw, self.deth = ntheta, detw, deth
        self.n1c, self.nthetac, self.dethc = n1c, nthetac, dethc
        self.cl_usfft1d = cfunc_usfft1d.cfunc_usfft1d(n0, n1c, n2, deth)
        self.cl_usfft2d = cfunc_usfft2d.cfunc_usfft2d(dethc, n1, n2, ntheta, detw, dethc)
        self.cl_fft2d = cfunc_fft2d.cfunc_fft2d(nthetac, detw, deth)

    def usfft1d_adj(self, out, inp, phi, stream):
        self.cl_usfft1d.adj(out, inp, phi, stream)

    def usfft2d_adj(self, out, inp, theta, phi, ind, stream):
        self.cl_usfft2d.adj(out, inp, theta, phi, ind, self.deth, stream)

    def fft2d_fwd(self, out, inp, stream):
        self.cl_fft2d.fwd(out, inp, stream)
