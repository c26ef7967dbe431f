"""``LpRec`` (src/tomocupy/reconstruction/lprec.py:292-335) over the native
``cfunc_lprec``: same constructor (angle check, grid sizes, grids built on the
host by :mod:`.lprec_grids` and kept alive on the device) and the same
``backprojection(obj, data, stream)``."""
from __future__ import annotations

import numpy as np
import torch

from .. import cfunc_lprec, cfunc_lprecfp16
from . import lprec_grids


class LpRec:
    def __init__(self, n, nproj, nz, theta, dtype, device="cuda"):
        th = np.asarray(theta.detach().cpu() if torch.is_tensor(theta) else theta)
        lprec_grids.check_angles(th, nproj)
        ntheta, nrho = lprec_grids.lp_sizes(n, nproj)
        P = lprec_grids.create_gl(n, nproj, ntheta, nrho)
        A = lprec_grids.create_adj(P)
        dev = torch.device(device)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
        # keep the grids alive for the native object's lifetime (it borrows them)
        self.grids = {
            "fz": torch.view_as_real(t(A.fZ)).contiguous(),
            "lp2p1": t(A.lp2p1), "lp2p2": t(A.lp2p2), "lp2p1w": t(A.lp2p1w),
            "lp2p2w": t(A.lp2p2w), "C2lp1": t(A.C2lp1), "C2lp2": t(A.C2lp2),
            "lpids": t(A.lpids), "wids": t(A.wids), "cids": t(A.cids),
        }
        # fZ stays float32 for both precisions (the fp16 variant only stores
        # the caller's sinograms and slices in fp16)
        mod =cfunc_lprecfp16 if dtype == "float16" else cfunc_lprec
        self.fslv = mod.cfunc_lprec(nproj, nz, n, ntheta, nrho)
        g = self.grids
        self.fslv.setgrids(g["fz"], g["lp2p1"], g["lp2p2"], g["lp2p1w"], g["lp2p2w"],
                           g["C2lp1"], g["C2lp2"], g["lpids"], g["wids"], g["cids"],
                           len(A.lpids), len(A.wids), len(A.cids))
        self.n, self.nproj, self.nz, self.ntheta, self.nrho = n, nproj, nz, ntheta, nrho
        self.dtype = dtype

    def backprojection(self, obj, data, stream=None):
        """obj [nz, n, n] <- lprec backprojection of data [nz, nproj, n] (data is overwritten)."""
        data = data.contiguous()
        self.fslv.backprojection(obj, data, stream)
        return obj
