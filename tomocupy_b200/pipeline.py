"""Device-resident reconstruction of one chunk of sinogram rows.

``SinoPipeline`` is the fused form of the reference's per-chunk sequence
(GPURec.recon_all, src/tomocupy/rec.py:161-179):

    proc_sino/proc_proj  ->  swapaxes  ->  fbp_filter_center  ->  backprojection

executed as native kernels on one stream:

 1. ``tcb_prep_rows``: uint16 frames -> dark/flat -> -log -> sinogram order,
    written straight into the edge-padded filter rows (one pass, no
    temporaries, no separate transpose or pad copies);
 2. ``tcb_filter_apply``: R2C -> per-slice complex spectrum -> C2R;
 3. fourierrec: ``tcb_fourierrec_pack`` (crop + complex pairing) and
    ``tcb_fourierrec_backprojection_slices`` (gridding, 2D FFT, deapodization,
    unpacking into the output slices);
    linerec: crop + ``tcb_linerec_backprojection``.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib, cfunc_filter, cfunc_fourierrec, cfunc_linerec
from .processing.proc_functions import in_dtype_code, prep_rows
from .reconstruction.backproj_functions import phase_weights, rfftfreq32
from .reconstruction.fbp_filter import calc_filter


class SinoPipeline:
    def __init__(self, n, nproj, ncz, theta, center, fbp_filter="parzen",
                 algorithm="fourierrec", minus_log=True, device="cuda", stripe=None):
        if algorithm not in ("fourierrec", "linerec", "lprec"):
            raise NotImplementedError(f"SinoPipeline: algorithm {algorithm!r}")
        if algorithm == "fourierrec" and ncz % 2:
            raise ValueError("fourierrec needs an even number of rows per chunk")
        self.device = torch.device(device)
        self.n, self.nproj, self.ncz = int(n), int(nproj), int(ncz)
        # lprec reconstructs about centre + 0.5, as BackprojFunctions sets it
        # (reconstruction/backproj_functions.py:70-71)
        self.center = float(center) + (0.5 if algorithm == "lprec" else 0.0)
        self.algorithm = algorithm
        self.minus_log = minus_log
        self.ne = 4 * self.n
        self.pad = self.ne // 2 - self.n // 2
        self.theta = torch.as_tensor(np.asarray(theta, dtype=np.float32), device=self.device)
        self.wfilter = torch.as_tensor(calc_filter(self.ne, fbp_filter), device=self.device)
        self.t = rfftfreq32(self.ne, self.device)
        self.rows = torch.empty((self.ncz, self.nproj, self.ne), dtype=torch.float32,
                                device=self.device)
        self.filter = cfunc_filter.cfunc_filter(self.nproj, self.ncz, self.ne)
        self._w_cache: dict = {}
        # optional Fourier-wavelet ring removal between dark/flat and -log
        # (ProcFunctions.proc_sino, proc_functions.py:140-160): stripe is
        # (sigma, wavelet, level)
        self.fw = None
        if stripe is not None:
            from .processing.remove_stripe import StripeFW
            sigma, wname, level = stripe
            self.fw = StripeFW(self.nproj, self.ncz, self.n, sigma, wname, level)
            self.sino = torch.zeros((self.ncz, self.fw.nproj_pad, self.n), dtype=torch.float32,
                                    device=self.device)
        if algorithm == "fourierrec":
            self.fr = cfunc_fourierrec.cfunc_fourierrec(self.nproj, self.ncz // 2, self.n,
                                                        self.theta)
            self.g = torch.empty((self.ncz // 2, self.nproj, self.n, 2), dtype=torch.float32,
                                 device=self.device)
        else:
            if algorithm == "linerec":
                self.lr = cfunc_linerec.cfunc_linerec(self.nproj, self.ncz, self.n, self.nproj,
                                                      self.ncz)
            else:
                from .reconstruction.lprec import LpRec
                self.lp = LpRec(self.n, self.nproj, self.ncz, theta, "float32",
                                device=self.device)
            self.crop = torch.empty((self.ncz, self.nproj, self.n), dtype=torch.float32,
                                    device=self.device)

    def weights(self, sht=None) -> torch.Tensor:
        """Per-slice filter spectra (cached for the zero shift)."""
        if sht is None:
            key = "zero"
            if key not in self._w_cache:
                z = torch.zeros(self.ncz, dtype=torch.float32, device=self.device)
                self._w_cache[key] = torch.view_as_real(
                    phase_weights(self.wfilter, self.t, self.center, z, self.n)).contiguous()
            return self._w_cache[key]
        sht = torch.as_tensor(sht, dtype=torch.float32, device=self.device).reshape(-1)
        return torch.view_as_real(
            phase_weights(self.wfilter, self.t, self.center, sht, self.n)).contiguous()

    def load_rows(self, data, dark0=None, flat0=None, z_lo=0, stream=None):
        """Fill the padded filter rows from a [nproj, nz, n] frame (or float) stack view."""
        nz = data.shape[1]
        assert nz <= self.ncz and data.shape[0] == self.nproj and data.shape[2] == self.n
        d0 = dark0[z_lo:z_lo + nz] if dark0 is not None else None
        f0 = flat0[z_lo:z_lo + nz] if flat0 is not None else None
        if self.fw is not None:
            fw = self.fw
            s = torch.cuda.current_stream() if stream is None else stream
            with torch.cuda.stream(s) if not isinstance(s, int) else _nullctx():
                self.sino.zero_()
            prep_rows(self.sino, data, d0, f0, darkflat=dark0 is not None, minus_log=False,
                      out_zstride=fw.nproj_pad * self.n, out_pstride=self.n,
                      out_poff=fw.poff, stream=stream)
            fw.apply_sino(self.sino, stream)
            src = self.sino[:nz, fw.poff:fw.poff + self.nproj].permute(1, 0, 2)
            prep_rows(self.rows, src, darkflat=False, minus_log=self.minus_log,
                      out_zstride=self.nproj * self.ne, out_pstride=self.ne, out_xoff=self.pad,
                      out_width=self.ne, edge_pad=True, stream=stream)
            return
        prep_rows(self.rows, data, d0, f0, darkflat=dark0 is not None,
                  minus_log=self.minus_log, out_zstride=self.nproj * self.ne,
                  out_pstride=self.ne, out_xoff=self.pad, out_width=self.ne, edge_pad=True,
                  stream=stream)

    def filter_and_backproject(self, out, sht=None, stream=None):
        """out [ncz, n, n] float32 (contiguous) from the loaded rows."""
        self.filter.filter(self.rows, self.weights(sht), stream)
        if self.algorithm == "fourierrec":
            self.fr.pack(self.g, self.rows, self.ne, self.pad, stream)
            self.fr.backprojection_slices(out, self.g, stream)
        else:
            s = torch.cuda.current_stream() if stream is None else stream
            with torch.cuda.stream(s) if not isinstance(s, int) else _nullctx():
                self.crop.copy_(self.rows[:, :, self.pad:self.pad + self.n])
                if self.algorithm == "linerec":
                    out.zero_()
            if self.algorithm == "linerec":
                self.lr.backprojection(out, self.crop, self.theta, math.pi / 2, 0, stream)
            else:
                self.lp.fslv.backprojection(out, self.crop, stream)
        return out

    def reconstruct(self, out, data, dark0=None, flat0=None, z_lo=0, sht=None, stream=None):
        self.load_rows(data, dark0, flat0, z_lo, stream)
        return self.filter_and_backproject(out, sht, stream)


class _nullctx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def copy2d_rows(dst: torch.Tensor, src: torch.Tensor, stream=None) -> None:
    """Async copy of a [a, b, c] view whose last two dims are contiguous per 'a' row."""
    assert dst.shape == src.shape and dst.dim() == 3
    a, b, c = src.shape
    es = src.element_size()
    assert src.stride(2) == 1 and dst.stride(2) == 1
    assert src.stride(1) == c and dst.stride(1) == c
    _lib.call("tcb_copy2d", dst.data_ptr(), dst.stride(0) * es, src.data_ptr(),
              src.stride(0) * es, b * c * es, a, _lib.stream_ptr(stream))
