"""Step-wise reconstruction: ``GPURecSteps.recon_steps_all``.

Mirrors ``GPURecSteps`` (src/tomocupy/rec_steps.py:64-243) and the
``BackprojParallel`` / ``BackprojLamFourierParallel`` back ends it selects
(reconstruction/backproj_parallel.py:57-422,
reconstruction/backproj_lamfourier_parallel.py:280-291):

* tomography (lamino_angle == 0), full: every sinogram chunk through the
  fused pipeline (same result as GPURec.recon_all);
* tomography, try: the centre sweep of GPURec.recon_try;
* laminography, fourierrec, full: the device-resident Fourier chain
  ``BackprojLamFourierParallel.rec_lam``;
* laminography, linerec (full / try / try_lamino): the projections are
  pre-processed and filtered once (the reference re-filters every
  projection chunk for every row chunk), then each block of output rows is
  backprojected over all angles with the tilted geometry.

The whole dataset is held in device memory between the steps (C3: 5 GB of
frames), replacing the reference's host-resident arrays and chunk copies.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .global_vars import args, params
from .pipeline import SinoPipeline
from .processing.proc_functions import (PHASE_METHODS, darkflat_stats, dezinger, dezinger_args,
                                        prep_rows, retrieve_phase)
from .reconstruction.backproj_functions import phase_weights, rfftfreq32
from .reconstruction.fbp_filter import calc_filter


class GPURecSteps:
    def __init__(self, cl_reader, cl_writer, device="cuda"):
        self.device = torch.device(device)
        self.cl_reader = cl_reader
        self.cl_writer = cl_writer
        if args.file_type not in ("standard", "double_fov"):
            raise NotImplementedError(f"file_type={args.file_type!r}")
        if args.file_type == "double_fov" and args.lamino_angle != 0:
            raise NotImplementedError("double-FOV laminography")
        if args.dtype not in ("float32", "float16", "mixed"):
            raise NotImplementedError(f"dtype={args.dtype!r}")

    # ------------------------------------------------------------ pre-processing
    def preprocessed(self):
        """[nproj, nz, n] float32 on the device after dark/flat, ring removal, -log
        (proc_sino_parallel + proc_proj_parallel, rec_steps.py:127-243)."""
        data, dark, flat = self.cl_reader.frames()
        dev = self.device
        data, dark, flat = data.to(dev), dark.to(dev), flat.to(dev)
        if args.pre_processing != "True":
            return data.to(torch.float32)
        dz = dezinger_args()
        if dz is not None:   # remove_outliers of data, darks and flats (proc_sino)
            data, dark, flat = dezinger(data, *dz), dezinger(dark, *dz), dezinger(flat, *dz)
        d0, f0, _ = darkflat_stats(dark, flat, args.bright_ratio)
        nproj, nz, n = data.shape
        out = torch.empty((nproj, nz, n), dtype=torch.float32, device=dev)
        stripe = args.remove_stripe_method in ("fw", "ti", "vo-all")
        phase = args.retrieve_phase_method in PHASE_METHODS
        rotate = float(args.rotate_proj_angle) != 0
        # -log comes last: after ring removal (proc_sino), phase retrieval and
        # rotation (proc_proj)
        late_log = stripe or phase or rotate
        prep_rows(out, data, d0, f0, darkflat=True,
                  minus_log=(args.minus_log == "True") and not late_log,
                  out_zstride=n, out_pstride=nz * n)
        if args.remove_stripe_method == "ti":
            from .processing.remove_stripe import remove_stripe_ti
            ncz = params.ncz
            for z0 in range(0, nz, ncz):
                part = out[:, z0:z0 + ncz].contiguous()
                out[:, z0:z0 + ncz] = remove_stripe_ti(part, args.ti_beta, args.ti_mask)
        elif args.remove_stripe_method == "vo-all":
            from .processing.remove_stripe import remove_all_stripe
            ncz = params.ncz
            for z0 in range(0, nz, ncz):
                part = out[:, z0:z0 + ncz].contiguous()
                out[:, z0:z0 + ncz] = remove_all_stripe(part, args.vo_all_snr,
                                                        args.vo_all_la_size,
                                                        args.vo_all_sm_size, args.vo_all_dim)
        elif stripe:
            from .processing.remove_stripe import remove_stripe_fw
            ncz = params.ncz
            for z0 in range(0, nz, ncz):
                out[:, z0:z0 + ncz] = remove_stripe_fw(out[:, z0:z0 + ncz].contiguous(),
                                                       args.fw_sigma, args.fw_filter,
                                                       args.fw_level)
        elif args.remove_stripe_method != "none":
            raise NotImplementedError(f"remove_stripe_method={args.remove_stripe_method!r}")
        if phase:
            retrieve_phase(out)
        if rotate:
            from .processing.proc_functions import rotate_proj
            out = rotate_proj(out, args.rotate_proj_angle, args.rotate_proj_order)
        if late_log and args.minus_log == "True":
            prep_rows(out, out, darkflat=False, minus_log=True, out_zstride=n,
                      out_pstride=nz * n)
        if args.file_type == "double_fov":
            out = self._pad360(out)
        return out

    def _pad360(self, out):
        """proc_proj's pad360 (proc_functions.py:109-124, 190-193) of every
        projection row: [nproj, nz, ni] -> [nproj, nz, 2 ni]."""
        from .processing.proc_functions import pad360, pad360_args
        return pad360(out, *pad360_args())

    # ------------------------------------------------------------------ driver
    def recon_steps_all(self):
        if args.lamino_angle == 0:
            return self._tomo()
        data = self.preprocessed()
        if args.reconstruction_algorithm == "fourierrec" and args.reconstruction_type == "full":
            from .reconstruction.backproj_lamfourier_parallel import BackprojLamFourierParallel
            u = BackprojLamFourierParallel(self.cl_writer, device=self.device).rec_lam(data)
            if args.dtype == "float16":
                u = self._out(u)
                self.cl_writer.rec = u.to(self.cl_writer.device)
            return u
        return self._lamino_linerec(data)

    def _tomo(self):
        from .rec import GPURec
        rec = GPURec(self.cl_reader, self.cl_writer, device=self.device)
        if (args.retrieve_phase_method in PHASE_METHODS or args.file_type == "double_fov"
                or float(args.rotate_proj_angle) != 0):
            # phase retrieval and rotation need whole projections, double-FOV
            # padding follows them: pre-process the resident dataset
            # (proc_sino + proc_proj), then backproject
            if args.reconstruction_type != "full":
                return rec.recon_try()   # proc_sino + proc_proj of each slice
            return rec.recon_preprocessed(self.preprocessed())
        if args.reconstruction_type == "full":
            return rec.recon_all()
        return rec.recon_try()

    @staticmethod
    def _out(vol):
        """The reference's dtype 'float16' returns float16 volumes."""
        if args.dtype == "float16" and vol.dtype != torch.float16:
            return vol.to(torch.float16)
        return vol

    # ------------------------------------------------- laminography with linerec
    def _filtered_projections(self, data):
        """fbp_filter_center of every projection (rows along the detector width),
        returned as [nz, nproj, n] (the layout linerec reads)."""
        from . import cfunc_filter
        nproj, nz, n = data.shape
        dev = self.device
        ne = 4 * n
        pad = ne // 2 - n // 2
        wf = torch.as_tensor(calc_filter(ne, args.fbp_filter), device=dev)
        t = rfftfreq32(ne, dev)
        ncp = max(1, min(nproj, params.ncproj))
        filt = cfunc_filter.cfunc_filter(nz, ncp, ne)
        w = torch.view_as_real(phase_weights(wf, t, params.center,
                                             torch.zeros(ncp, device=dev), n)).contiguous()
        rows = torch.empty((ncp, nz, ne), dtype=torch.float32, device=dev)
        out = torch.empty((nz, nproj, n), dtype=torch.float32, device=dev)
        for st in range(0, nproj, ncp):
            end = min(nproj, st + ncp)
            rows.zero_()
            # chunk [end-st, nz, n] as "[nproj=nz rows][nz=projections]" -> rows [proj][z][ne]
            prep_rows(rows, data[st:end].permute(1, 0, 2), darkflat=False, minus_log=False,
                      out_zstride=nz * ne, out_pstride=ne, out_xoff=pad, out_width=ne,
                      edge_pad=True)
            filt.filter(rows, w, None)
            out[:, st:end] = rows[:end - st, :, pad:pad + n].permute(1, 0, 2)
        return out

    def _lamino_linerec(self, data):
        from .reconstruction.linerec import LineRec
        nproj, nz, n = data.shape
        dev = self.device
        g = self._filtered_projections(data)
        theta = torch.as_tensor(np.asarray(params.theta, dtype=np.float32), device=dev)
        ncz = params.ncz
        lr = LineRec(theta, nproj, nproj, nz, ncz, n, "float32")  # filtered rows are fp32
        if args.reconstruction_type == "full":
            rh = params.rh
            vol = torch.zeros((rh, n, n), dtype=torch.float32, device=dev)
            f = torch.zeros((ncz, n, n), dtype=torch.float32, device=dev)
            for r0 in range(0, rh, ncz):
                f.zero_()
                lr.backprojection(f, g, None, theta, args.lamino_angle,
                                  r0 + args.lamino_start_row)
                vol[r0:r0 + ncz] = f[:min(ncz, rh - r0)]
            vol = self._out(vol)
            self.cl_writer.rec = vol
            return vol
        results = {}
        shifts = torch.as_tensor(params.shift_array, dtype=torch.float32, device=dev)
        for id_slice in params.id_slices:
            for k in range(params.nschunk):
                lk = int(params.lschunk[k])
                sh = torch.zeros(ncz, dtype=torch.float32, device=dev)
                sh[:lk] = shifts[k * ncz:k * ncz + lk]
                f = torch.zeros((ncz, n, n), dtype=torch.float32, device=dev)
                if args.reconstruction_type == "try":
                    lr.backprojection_try(f, g, sh, None, theta, args.lamino_angle, int(id_slice))
                else:
                    lr.backprojection_try_lamino(f, g, sh, None, theta, args.lamino_angle,
                                                 int(id_slice))
                for kk in range(lk):
                    self.cl_writer.write_data_try(f[kk], params.save_centers[k * ncz + kk],
                                                  id_slice)
                    results[(int(id_slice), float(params.save_centers[k * ncz + kk]))] = f[kk]
        return results
