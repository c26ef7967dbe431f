"""Method selection and the centred FBP filter step.

Mirrors ``BackprojFunctions`` (src/tomocupy/reconstruction/backproj_functions.py:47-109):
it reads ``params`` / ``args`` the same way, picks the backprojector, sets
``ne = 4n`` (next power of two for float16), builds the filter spectrum, and
``fbp_filter_center`` edge-pads to ``ne``, multiplies by the per-slice
centre-shift phase ramp and filters.  Torch tensors stand in for CuPy arrays.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ..global_vars import args, params
from . import fbp_filter, fourierrec, linerec


def phase_weights(wfilter: torch.Tensor, t: torch.Tensor, center: float, sht: torch.Tensor,
                  n: int) -> torch.Tensor:
    """w[z, k] = wfilter[k] * exp(-2*pi*i*(-center + sht[z] + n/2) * t[k]) in complex64.

    Operation order of backproj_functions.py:103-104: the real shift is formed
    in float32, multiplied by the complex64 constant -2*pi*i (an exact float32
    doubling of pi), then by t, exponentiated and scaled by the filter.
    """
    a = (-center + sht.to(torch.float32)) + n / 2          # float32 [nz]
    ci = np.float32(-2.0) * np.float32(math.pi)            # imag of -2*complex64(pi*1j)
    phase = (a * float(ci))[:, None] * t[None, :]          # float32 [nz, nc]
    return torch.complex(wfilter * torch.cos(phase), wfilter * torch.sin(phase))


def rfftfreq32(ne: int, device) -> torch.Tensor:
    """cupy.fft.rfftfreq(ne).astype('float32'): arange(0, ne//2+1)/ne in float64."""
    return (torch.arange(0, ne // 2 + 1, dtype=torch.float64, device=device) / ne).to(
        torch.float32)


class BackprojFunctions:
    def __init__(self, device=None):
        self.device = torch.device(device or "cuda")
        params.ne = 4 * params.n
        if args.dtype == "float16":
            # power of 2 for float16
            params.ne = 2 ** int(math.ceil(math.log2(params.ne)))

        theta = torch.as_tensor(np.asarray(params.theta, dtype=np.float32), device=self.device)

        if args.lamino_angle != 0:
            self.cl_rec = linerec.LineRec(theta, params.nproj, params.ncproj, params.nz,
                                          params.ncz, params.n, args.dtype)
            self.cl_filter = fbp_filter.FBPFilter(params.ne, params.ncproj, params.nz, args.dtype)
        else:
            if args.reconstruction_algorithm == "fourierrec":
                self.cl_rec = fourierrec.FourierRec(params.n, params.nproj, params.ncz, theta,
                                                    args.dtype)
            elif args.reconstruction_algorithm == "lprec":
                from . import lprec
                params.centeri += 0.5  # consistency with the Fourier-based method
                params.center += 0.5
                self.cl_rec = lprec.LpRec(params.n, params.nproj, params.ncz, theta, args.dtype)
            elif args.reconstruction_algorithm == "linerec":
                self.cl_rec = linerec.LineRec(theta, params.nproj, params.nproj, params.ncz,
                                              params.ncz, params.n, args.dtype)
            else:
                raise ValueError(f"unknown algorithm {args.reconstruction_algorithm!r}")
            self.cl_filter = fbp_filter.FBPFilter(params.ne, params.nproj, params.ncz, args.dtype)

        self.wfilter = torch.as_tensor(self.cl_filter.calc_filter(args.fbp_filter),
                                       device=self.device)
        self.pad = params.ne // 2 - params.n // 2
        self.t = rfftfreq32(params.ne, self.device)
        if args.lamino_angle != 0:
            nz_filter, ntheta_filter = params.nz, params.ncproj
        else:
            nz_filter, ntheta_filter = params.ncz, params.nproj
        tdt = torch.float16 if args.dtype == "float16" else torch.float32
        self._tmp = torch.empty((nz_filter, ntheta_filter, params.ne), dtype=tdt,
                                device=self.device)

    def fbp_filter_center(self, data, sht=0):
        """FBP filtering of [nz, nproj, n] rows with the rotation-centre shift (in place)."""
        nz = data.shape[0]
        n = params.n
        tmp = self._tmp[:nz]
        tmp[:, :, self.pad:self.pad + n] = data
        tmp[:, :, :self.pad] = data[:, :, :1]
        tmp[:, :, self.pad + n:] = data[:, :, -1:]
        if not torch.is_tensor(sht):
            sht = torch.full((nz,), float(sht), dtype=torch.float32, device=data.device)
        sht = sht.reshape(-1)[:nz] if sht.numel() >= nz else sht.reshape(-1)
        w = phase_weights(self.wfilter, self.t, params.center, sht, n)
        self.cl_filter.filter(tmp, w, torch.cuda.current_stream())
        data[:] = tmp[:, :, self.pad:self.pad + n]
        return data
