"""Laminographic reconstruction by the Fourier chain, device resident.

Mirrors ``BackprojLamFourierParallel`` (src/tomocupy/reconstruction/
backproj_lamfourier_parallel.py:57-304): the same three stages

  1. per chunk of ``nthetac`` projections: FBP filter along detector rows and
     2D R2C FFT  ->  S1 [ntheta, deth, detw/2+1]
  2. per chunk of ``dethc`` frequency rows: adjoint 2D USFFT
     ->  S2 [n1, deth/2+1, n2]
  3. per chunk of ``n1c`` rows: adjoint 1D USFFT along the height
     ->  S3 [n1, rh, n2]
  4. transpose  ->  volume [rh, n1, n2]

but the intermediates stay in HBM (C3: 5.0 + 4.3 + 2.1 GB), so the
reference's device->pinned->host->pinned->device round trips between stages
and its host-side packing of the conjugate-mirrored rows disappear: the
usfft2d stage reads S1 in place (``cfunc_usfft2d.adj_rows``).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .. import _lib
from ..global_vars import args, params
from ..processing.proc_functions import prep_rows
from ..reconstruction.backproj_functions import rfftfreq32
from . import fbp_filter, lamfourierrec


class BackprojLamFourierParallel:
    def __init__(self, cl_writer=None, device="cuda"):
        self.device = torch.device(device)
        self.n0 = params.rh
        self.n1 = params.n
        self.n2 = params.n
        self.ntheta = params.nproj
        self.nthetac = params.ncproj
        self.detw = params.n
        self.deth = params.nz
        self.n1c = params.ncz
        self.dethc = params.ncz
        self.center = params.center
        self.ne = 4 * self.detw
        self.cl_lamfourier = lamfourierrec.LamFourierRec(
            self.n0, self.n1, self.n2, self.ntheta, self.detw, self.deth, self.n1c,
            self.nthetac, self.dethc)
        # filter applied along the rows of each projection (not sinograms)
        self.cl_filter = fbp_filter.FBPFilter(self.ne, self.deth, self.nthetac, args.dtype)
        self.wfilter = torch.as_tensor(self.cl_filter.calc_filter(args.fbp_filter),
                                       device=self.device)
        self.pad = self.ne // 2 - self.detw // 2
        self.t = rfftfreq32(self.ne, self.device)
        self._rows = torch.empty((self.nthetac, self.deth, self.ne), dtype=torch.float32,
                                 device=self.device)
        self._crop = torch.empty((self.nthetac, self.deth, self.detw), dtype=torch.float32,
                                 device=self.device)
        self.cl_writer = cl_writer
        self.rec_fun = self.rec_lam

    def _weights(self, nthetac):
        # backproj_lamfourier_parallel.py:270-271: (-2*pi*i * t) * (-center + sht + n2/2)
        ci = float(np.float32(-2.0) * np.float32(math.pi))
        a = torch.full((nthetac, 1), -self.center, dtype=torch.float32,
                       device=self.device) + self.n2 / 2
        phase = (self.t * ci)[None, :] * a
        w = torch.complex(self.wfilter * torch.cos(phase), self.wfilter * torch.sin(phase))
        return torch.view_as_real(w).contiguous()

    def rec_lam(self, data, stream=None):
        """data [ntheta, deth, detw] float32 (host or device) -> volume [rh, n1, n2]."""
        dev = self.device
        phi = math.pi / 2 + params.lamino_angle / 180 * math.pi
        theta = torch.as_tensor(np.asarray(params.theta, dtype=np.float32), device=dev)
        nthetac, deth, detw = self.nthetac, self.deth, self.detw
        w = self._weights(nthetac)
        # fp16 storage of the two stage arrays (fp32 arithmetic) in mixed precision
        half = args.dtype in ("mixed", "float16")  # fp16 storage of the stage arrays
        sdt = torch.float16 if half else torch.float32
        prec = _lib.TCB_FLOAT16 if half else _lib.TCB_FLOAT32
        nrow = deth // 2 + 1
        # fp16 stage arrays carry power-of-two scales: inv1 per angle, inv2 per
        # frequency row (written by usfft2d), so values stay in fp16's normal range
        inv1 = torch.ones(self.ntheta, dtype=torch.float32, device=dev) if half else None
        inv2 = torch.ones(nrow, dtype=torch.float32, device=dev) if half else None
        self.cl_lamfourier.cl_usfft2d.set_storage(prec, inv1, inv2)
        self.cl_lamfourier.cl_usfft1d.set_storage(prec, inv2)
        s1 = torch.empty((self.ntheta, deth, detw // 2 + 1, 2), dtype=sdt, device=dev)
        g1 = torch.empty((nthetac, deth, detw // 2 + 1), dtype=torch.complex64, device=dev)
        # stage 1
        for st in range(0, self.ntheta, nthetac):
            end = min(self.ntheta, st + nthetac)
            chunk = data[st:end]
            if chunk.device != dev:
                chunk = chunk.to(dev, non_blocking=True)
            if end - st < nthetac:
                self._rows.zero_()
            prep_rows(self._rows, chunk.permute(1, 0, 2), darkflat=False, minus_log=False,
                      out_zstride=deth * self.ne, out_pstride=self.ne, out_xoff=self.pad,
                      out_width=self.ne, edge_pad=True, stream=stream)
            self.cl_filter.fslv.filter(self._rows, w, stream)
            self._crop.copy_(self._rows[:, :, self.pad:self.pad + detw])
            self.cl_lamfourier.fft2d_fwd(g1, self._crop, stream)
            gr = torch.view_as_real(g1[:end - st])
            if half:
                _, e = torch.frexp(gr.abs().amax())
                sig = torch.ldexp(torch.ones((), device=dev), 14 - e)
                s1[st:end] = gr * sig
                inv1[st:end] = 1.0 / sig
            else:
                s1[st:end] = gr
        # stage 2
        s2 = torch.empty((self.n1, nrow, self.n2, 2), dtype=sdt, device=dev)
        for st in range(0, nrow, self.dethc):
            nr = min(self.dethc, nrow - st)
            self.cl_lamfourier.cl_usfft2d.adj_rows(s2, s1, theta, phi, st, nr, deth, stream)
        del s1
        # stage 3
        s3 = torch.empty((self.n1, self.n0, self.n2), dtype=torch.float32, device=dev)
        o1 = torch.empty((self.n1c, self.n0, self.n2), dtype=torch.float32, device=dev)
        gin = torch.zeros((self.n1c, nrow, self.n2, 2), dtype=sdt, device=dev)
        for st in range(0, self.n1, self.n1c):
            end = min(self.n1, st + self.n1c)
            if end - st == self.n1c:
                self.cl_lamfourier.usfft1d_adj(s3[st:end], s2[st:end], phi, stream)
            else:
                gin[:end - st] = s2[st:end]
                self.cl_lamfourier.usfft1d_adj(o1, gin, phi, stream)
                s3[st:end] = o1[:end - st]
        # stage 4: copyTransposed
        u = s3.permute(1, 0, 2).contiguous()
        if self.cl_writer is not None:
            self.cl_writer.allocate(u.shape[0], self.n1)  # square slices
            self.cl_writer.rec = u if self.cl_writer.device == dev else u.to(self.cl_writer.device)
        return u
