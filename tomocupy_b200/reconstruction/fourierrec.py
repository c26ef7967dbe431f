"""``FourierRec`` (src/tomocupy/reconstruction/fourierrec.py:46-68) over the native
``cfunc_fourierrec``.  Slices ``k`` and ``k + nz/2`` travel as the real and
imaginary parts of one complex sinogram; the native entry point unpacks the
result straight into the two real output slices, so the reference's two
reorganisation copies of the output disappear."""
from __future__ import annotations

import torch

from .. import cfunc_fourierrec, cfunc_fourierrecfp16


class FourierRec:
    """Backprojection by the Fourier-based method."""

    def __init__(self, n, nproj, nz, theta, dtype):
        self.theta = theta  # keep theta alive, as the reference does
        self.nz = nz
        self.n = n
        self.nproj = nproj
        self.dtype = dtype
        mod = cfunc_fourierrecfp16 if dtype == "float16" else cfunc_fourierrec
        self.fslv = mod.cfunc_fourierrec(nproj, nz // 2, n, self.theta)

    def backprojection(self, obj, data, stream):
        """obj [nz, n, n] <- FBP of the filtered sinograms data [nz, nproj, n]."""
        h = self.nz // 2
        cdt = torch.float16 if self.dtype == "float16" else torch.float32
        # complex pairing (fourierrec.py:63-64): real = data[:h], imag = data[h:]
        g = torch.stack((data[:h], data[h:]), dim=-1).to(cdt).contiguous()
        if obj.is_contiguous() and obj.dtype == cdt:
            self.fslv.backprojection_slices(obj, g, stream)
        else:
            out = torch.empty((self.nz, self.n, self.n), dtype=cdt, device=obj.device)
            self.fslv.backprojection_slices(out, g, stream)
            obj[:] = out
        return obj
