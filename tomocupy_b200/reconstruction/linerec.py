"""``LineRec`` (src/tomocupy/reconstruction/linerec.py:44-85) over the native
``cfunc_linerec``: same arguments, same accumulate semantics (``f`` is
zeroed only when the default angle set is used)."""
from __future__ import annotations

import math

import torch

from .. import cfunc_linerec, cfunc_linerecfp16


class LineRec:
    """Backprojection by summation over lines."""

    def __init__(self, theta, nproj, ncproj, nz, ncz, n, dtype):
        self.nproj = nproj
        self.ncproj = ncproj
        self.nz = nz
        self.ncz = ncz
        self.n = n
        self.dtype = dtype
        self.theta = torch.as_tensor(theta, dtype=torch.float32, device="cuda")
        mod = cfunc_linerecfp16 if dtype == "float16" else cfunc_linerec
        self.fslv = mod.cfunc_linerec(nproj, nz, n, ncproj, ncz)

    def backprojection(self, f, data, stream=None, theta=(), lamino_angle=0, sz=0):
        if len(theta) == 0:
            theta = self.theta
            f[:] = 0
        phi = math.pi / 2 + lamino_angle / 180 * math.pi
        self.fslv.backprojection(f, data.contiguous(), theta.contiguous(), phi, sz, stream)

    def backprojection_try(self, f, data, sh, stream=None, theta=(), lamino_angle=0, sz=0):
        if len(theta) == 0:
            theta = self.theta
        phi = math.pi / 2 + lamino_angle / 180 * math.pi
        self.fslv.backprojection_try(f, data.contiguous(), theta.contiguous(),
                                     sh.to(torch.float32).contiguous(), phi, sz, stream)

    def backprojection_try_lamino(self, f, data, sh, stream=None, theta=(), lamino_angle=0,
                                  sz=0):
        if len(theta) == 0:
            theta = self.theta
        # (cp.pi/2 + (angle + sh)/180*cp.pi) with sh float32: Python scalars do not
        # promote, so every step is float32
        phi = (math.pi / 2 + (lamino_angle + sh.to(torch.float32)) / 180 * math.pi).contiguous()
        self.fslv.backprojection_try_lamino(f, data.contiguous(), theta.contiguous(), phi, sz,
                                            stream)
