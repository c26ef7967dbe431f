"""Chunked reconstruction drivers: ``GPURec.recon_all`` and ``GPURec.recon_try``.

Mirrors ``GPURec`` (src/tomocupy/rec.py:62-275).  The reference's conveyor
(read queue -> pinned staging -> H2D on stream1 -> compute on stream2 ->
D2H on stream3, with a host ``synchronize()`` of every stream each
iteration) becomes a device-side dependency graph: each chunk's H2D,
compute and D2H are ordered by CUDA events only, buffers are double
buffered, and the host blocks once at the end.  Slabs of the host stack are
moved with one strided 2D copy each (no host repacking).  Dark/flat means
are computed once for all rows and stay resident.

``recon_device`` is the same reconstruction with the whole input already in
device memory (no host traffic at all).
"""
from __future__ import annotations

import numpy as np
import torch

from .global_vars import args, params
from .pipeline import SinoPipeline, copy2d_rows
from .processing.proc_functions import (PHASE_METHODS, darkflat_stats, dezinger, dezinger_args,
                                        pad360_args, prep_rows, retrieve_phase, rotate_proj)


def _supported():
    if args.remove_stripe_method not in ("none", "fw", "ti", "vo-all"):
        raise NotImplementedError(
            f"remove_stripe_method={args.remove_stripe_method!r} is not part of tomocupy_b200")
    if args.file_type not in ("standard", "double_fov"):
        raise NotImplementedError(f"file_type={args.file_type!r}")
    if not 0 <= int(args.binning) <= 4:
        raise NotImplementedError("binning above 4")
    if args.dtype not in ("float32", "float16", "mixed"):
        raise NotImplementedError(f"dtype={args.dtype!r}")


def _stripe_args():
    """The pipeline's ring-removal argument for remove_stripe_method, else None."""
    if args.remove_stripe_method == "fw":
        return (float(args.fw_sigma), args.fw_filter, int(args.fw_level))
    if args.remove_stripe_method == "ti":
        return ("ti", float(args.ti_beta), float(args.ti_mask))
    if args.remove_stripe_method == "vo-all":
        return ("vo-all", float(args.vo_all_snr), int(args.vo_all_la_size),
                int(args.vo_all_sm_size), int(args.vo_all_dim))
    return None


_pad360_args = pad360_args


def _rotate():
    return float(args.rotate_proj_angle) != 0


def _proj_chunk_ops():
    """proc_proj steps that recon_all runs on each chunk's projections (phase
    retrieval, rotation) before the pipeline's -log."""
    return args.retrieve_phase_method in PHASE_METHODS or _rotate()


class GPURec:
    """Tomographic reconstruction by sinogram chunks on one GPU."""

    def __init__(self, cl_reader, cl_writer, device="cuda"):
        _supported()
        self.device = torch.device(device)
        self.cl_reader = cl_reader
        self.cl_writer = cl_writer
        self._pipe = None
        self.sweep = None
        self.stream1 = torch.cuda.Stream(self.device)
        self.stream2 = torch.cuda.Stream(self.device)
        self.stream3 = torch.cuda.Stream(self.device)

    @property
    def precision(self) -> str:
        """'mixed' (fp16 weights and values on the tensor cores, fp32
        accumulation) for dtype 'mixed' and, with fourierrec, for the
        reference's dtype 'float16' (its cfunc_*fp16 operators grid in fp16);
        'float32' otherwise."""
        if args.dtype == "mixed":
            return "mixed"
        if args.dtype == "float16" and args.reconstruction_algorithm == "fourierrec":
            return "mixed"
        return "float32"

    @staticmethod
    def out_dtype() -> str:
        """Output slices: float16 for the reference's dtype 'float16' (its
        reconstruction arrays are float16), else args.out_dtype."""
        return "float16" if args.dtype == "float16" else args.out_dtype

    @property
    def pipe(self) -> SinoPipeline:
        """The chunk pipeline (built on first use; try-centre sweeps do not need it)."""
        if self._pipe is None:
            # with phase retrieval or rotation the chunk's outlier removal and
            # ring removal run before them (_phase_chunk), not in the pipeline
            proj_ops = _proj_chunk_ops()
            stripe = None if proj_ops else _stripe_args()
            self._pipe = SinoPipeline(params.n, params.nproj, params.ncz, params.theta,
                                      params.center, args.fbp_filter,
                                      args.reconstruction_algorithm,
                                      minus_log=args.minus_log == "True", device=self.device,
                                      stripe=stripe, precision=self.precision,
                                      out_dtype=self.out_dtype(),
                                      mixed_filter=args.mixed_filter,
                                      dezinger=None if proj_ops else dezinger_args(),
                                      ni=params.ni,
                                      pad360=_pad360_args())
        return self._pipe

    # ------------------------------------------------------------------ helpers
    def _stats(self, dark, flat, stream):
        """dark0, flat0 and (flat_linear) flat1 of darkflat_correction
        (proc_functions.py:55-74), after outlier removal of the darks and flats."""
        dz = dezinger_args()
        if dz is not None:   # proc_sino cleans darks and flats too (proc_functions.py:146-148)
            dark = dezinger(dark, *dz, stream=stream)
            flat = dezinger(flat, *dz, stream=stream)
        return darkflat_stats(dark, flat, args.bright_ratio, args.flat_linear == "True", stream)

    # ------------------------------------------------------------------ full
    def recon_preprocessed(self, data):
        """Reconstruct every slice from pre-processed float32 projections
        [nproj, nz, n] on the device (the step driver after proc_sino and
        proc_proj: filter and backprojection only); results go to cl_writer."""
        ncz, n, nz = params.ncz, params.n, params.nz
        assert data.dtype == torch.float32 and tuple(data.shape) == (params.nproj, nz, n)
        pipe = SinoPipeline(n, params.nproj, ncz, params.theta, params.center, args.fbp_filter,
                            args.reconstruction_algorithm, minus_log=False, device=self.device,
                            stripe=None, precision=self.precision, out_dtype=self.out_dtype(),
                            mixed_filter=args.mixed_filter)
        rec_out = self.cl_writer.allocate(nz, n)
        out = torch.empty((ncz, n, n), dtype=pipe.out_dtype, device=self.device)
        for k in range(params.nzchunk):
            z0, lz = k * ncz, int(params.lzchunk[k])
            if lz < ncz:
                pipe.clear_rows(lz)
            pipe.reconstruct(out, data[:, z0:z0 + lz])
            rec_out[z0:z0 + lz].copy_(out[:lz])
        torch.cuda.synchronize(self.device)
        return rec_out

    def recon_all(self):
        """Reconstruct every slice; results go to ``cl_writer`` (host or device)."""
        phase = _proj_chunk_ops()
        data, dark, flat = self.cl_reader.frames()
        ncz, n, nz, nproj = params.ncz, params.n, params.nz, params.nproj
        dev = self.device
        rec_out = self.cl_writer.allocate(nz, n)
        s1, s2, s3 = self.stream1, self.stream2, self.stream3
        cur = torch.cuda.current_stream(dev)
        s1.wait_stream(cur)
        s2.wait_stream(cur)
        s3.wait_stream(cur)
        # dark/flat: one upload, statistics for all rows, resident
        with torch.cuda.stream(s1):
            dark_d = dark.to(dev, non_blocking=True)
            flat_d = flat.to(dev, non_blocking=True)
        s2.wait_stream(s1)
        with torch.cuda.stream(s2):
            dark0, flat0, flat1 = self._stats(dark_d, flat_d, s2)
        host_in = data.device.type == "cpu"
        host_out = rec_out.device.type == "cpu"
        dbuf = [torch.empty((nproj, ncz, data.shape[2]), dtype=data.dtype, device=dev)
                for _ in range(2)]
        odt = self.pipe.out_dtype
        if rec_out.dtype != odt:
            raise ValueError(f"writer dtype {rec_out.dtype} != output dtype {odt} (args.out_dtype)")
        rbuf = [torch.empty((ncz, n, n), dtype=odt, device=dev) for _ in range(2)]
        h2d_done = [torch.cuda.Event() for _ in range(2)]
        comp_done = [torch.cuda.Event() for _ in range(2)]
        d2h_done = [torch.cuda.Event() for _ in range(2)]
        nchunk = params.nzchunk
        for k in range(nchunk):
            b = k % 2
            z0 = k * ncz
            lz = int(params.lzchunk[k])
            # H2D of the slab (waits until compute of chunk k-2 released dbuf[b])
            if host_in:
                with torch.cuda.stream(s1):
                    if k >= 2:
                        s1.wait_event(comp_done[b])
                    copy2d_rows(dbuf[b][:, :lz], data[:, z0:z0 + lz], s1)
                    h2d_done[b].record(s1)
                src = dbuf[b][:, :lz]
            else:
                src = data[:, z0:z0 + lz]
            with torch.cuda.stream(s2):
                if host_in:
                    s2.wait_event(h2d_done[b])
                if k >= 2 and host_out:
                    s2.wait_event(d2h_done[b])
                out = rbuf[b] if (host_out or lz < ncz) else rec_out[z0:z0 + ncz]
                if lz < ncz:  # rows of the previous chunk must not pair with this one's
                    self.pipe.clear_rows(lz, s2)
                if phase:
                    self.pipe.reconstruct(out, self._phase_chunk(src, dark0, flat0, z0, s2,
                                                                 flat1),
                                          None, None, z_lo=z0, stream=s2)
                else:
                    self.pipe.reconstruct(out, src, dark0, flat0, z_lo=z0, stream=s2,
                                          flat1=flat1)
                if not host_out and lz < ncz:
                    rec_out[z0:z0 + lz].copy_(out[:lz])
                comp_done[b].record(s2)
            if host_out:
                with torch.cuda.stream(s3):
                    s3.wait_event(comp_done[b])
                    rec_out[z0:z0 + lz].copy_(rbuf[b][:lz], non_blocking=True)
                    d2h_done[b].record(s3)
        cur.wait_stream(s1)
        cur.wait_stream(s2)
        cur.wait_stream(s3)
        torch.cuda.synchronize(dev)
        return rec_out

    # ------------------------------------------------------------------ try
    def recon_try(self):
        """Reconstruct slice(s) ``params.id_slices`` for every centre in ``params.shift_array``.

        The sweep over all centres is one CUDA graph (TryCenterSweep), recorded
        once and replayed for each requested slice.
        """
        from .trycenter import TryCenterSweep
        if args.reconstruction_algorithm != "fourierrec":
            return self._recon_try_chunks()
        data, dark, flat = self.cl_reader.frames()
        dev = self.device
        proj_ops = _proj_chunk_ops()
        if self.sweep is None:
            self.sweep = TryCenterSweep(params.n, params.nproj, params.theta, params.center,
                                        params.shift_array, args.fbp_filter, self.precision,
                                        params.ncz, device=dev,
                                        minus_log=args.minus_log == "True",
                                        mixed_filter=args.mixed_filter, ni=params.ni,
                                        pad360=_pad360_args(),
                                        stripe=None if proj_ops else _stripe_args())
        sw = self.sweep
        for id_slice in params.id_slices:
            z = int(id_slice)
            row = data[:, z:z + 1].to(dev)
            d0, f0, f1 = self._stats(dark[:, z:z + 1].to(dev), flat[:, z:z + 1].to(dev), None)
            if proj_ops:
                # proc_sino then proc_proj on the one-row slice, as the
                # reference's recon_try does (rec.py:224-225): the image height
                # of phase retrieval and rotation is 1
                sw.load(self._phase_chunk(row, d0, f0, 0, None, f1, chunk_height=False))
            else:
                if dezinger_args() is not None:
                    row = dezinger(row, *dezinger_args())
                sw.load(row, d0, f0, f1)
            if sw.graph is None:
                sw.capture()
            out = sw.run()
            for k in range(sw.S):
                self.cl_writer.write_data_try(out[k], params.save_centers[k], id_slice)
        torch.cuda.synchronize(dev)

    def _phase_chunk(self, src, dark0, flat0, z0, stream, flat1=None, chunk_height=True):
        """proc_sino + proc_proj's phase step on one sinogram chunk, as the
        reference's recon_all runs them (rec.py:170-173): outlier removal,
        dark/flat, ring removal, then phase retrieval and rotation of the
        chunk's projections (its rows are the image height); -log (and
        double-FOV padding) follow in the pipeline."""
        nproj, lz, n = src.shape
        dz = dezinger_args()
        if dz is not None:  # proc_sino: outliers of the raw frames first (proc_functions.py:146-148)
            zb = getattr(self, "_phase_zbuf", None)
            if zb is None or zb.dtype != src.dtype or zb.numel() < nproj * lz * n:
                zb = self._phase_zbuf = torch.empty(nproj * params.ncz * n, dtype=src.dtype,
                                                    device=self.device)
            src = dezinger(src, *dz, out=zb[:nproj * lz * n].view(nproj, lz, n), stream=stream)
        buf = getattr(self, "_phase_buf", None)
        if buf is None or buf.numel() < nproj * lz * n:
            buf = self._phase_buf = torch.empty(nproj * params.ncz * n, dtype=torch.float32,
                                                device=self.device)
        tmp = buf[:nproj * lz * n].view(nproj, lz, n)
        prep_rows(tmp, src, dark0[z0:z0 + lz], flat0[z0:z0 + lz],
                  flat1[z0:z0 + lz] if flat1 is not None else None, darkflat=True,
                  minus_log=False, flat_linear=flat1 is not None, out_zstride=n,
                  out_pstride=lz * n, stream=stream)
        with torch.cuda.stream(stream):
            if args.remove_stripe_method == "fw":
                from .processing.remove_stripe import remove_stripe_fw
                tmp.copy_(remove_stripe_fw(tmp, args.fw_sigma, args.fw_filter, args.fw_level))
            elif args.remove_stripe_method == "ti":
                from .processing.remove_stripe import remove_stripe_ti
                remove_stripe_ti(tmp, args.ti_beta, args.ti_mask)
            elif args.remove_stripe_method == "vo-all":
                from .processing.remove_stripe import remove_all_stripe
                remove_all_stripe(tmp, args.vo_all_snr, args.vo_all_la_size,
                                  args.vo_all_sm_size, args.vo_all_dim)
            retrieve_phase(tmp)
        if _rotate() and not chunk_height:
            # a try-centre slice is rotated at its own height
            out = torch.empty_like(tmp)
            rotate_proj(tmp, args.rotate_proj_angle, args.rotate_proj_order, out=out,
                        stream=stream)
            return out
        if _rotate():
            # the reference rotates its chunk buffer of ncz rows: a partial
            # chunk is rotated at that height with zero rows below it
            rb = getattr(self, "_rot_buf", None)
            if rb is None or rb.shape[1] != nproj * params.ncz * n:
                rb = self._rot_buf = torch.empty((2, nproj * params.ncz * n),
                                                 dtype=torch.float32, device=self.device)
            rin = rb[0].view(nproj, params.ncz, n)
            rout = rb[1].view(nproj, params.ncz, n)
            if lz < params.ncz:
                with torch.cuda.stream(stream):
                    rin.zero_()
                    rin[:, :lz].copy_(tmp)
                src_rot = rin
            else:
                src_rot = tmp
            rotate_proj(src_rot, args.rotate_proj_angle, args.rotate_proj_order, out=rout,
                        stream=stream)
            return rout[:, :lz]
        return tmp

    def _recon_try_chunks(self):
        """Try-centre reconstruction with lprec or linerec, as the reference's
        recon_try does it (rec.py:210-275): the pre-processed slice tiled ncz
        times, each copy filtered with its own centre shift, one backprojection
        per chunk of ncz shifts."""
        data, dark, flat = self.cl_reader.frames()
        dev, ncz, n = self.device, params.ncz, params.n
        pipe = self.pipe
        shifts = np.asarray(params.shift_array, dtype=np.float32)
        out = torch.empty((ncz, n, n), dtype=pipe.out_dtype, device=dev)
        proj_ops = _proj_chunk_ops()
        for id_slice in params.id_slices:
            z = int(id_slice)
            row = data[:, z:z + 1].to(dev)
            d0, f0, f1 = self._stats(dark[:, z:z + 1].to(dev), flat[:, z:z + 1].to(dev), None)
            if proj_ops:   # proc_sino + proc_proj on the slice (rec.py:224-225)
                row = self._phase_chunk(row, d0, f0, 0, None, f1, chunk_height=False)
                d0 = f0 = f1 = None
            elif dezinger_args() is not None:
                row = dezinger(row, *dezinger_args())
            for k0 in range(0, shifts.size, ncz):
                cnt = min(ncz, shifts.size - k0)
                sht = np.zeros(ncz, dtype=np.float32)
                sht[:cnt] = shifts[k0:k0 + cnt]
                pipe.load_rows(row, d0, f0, 0, flat1=f1)
                pipe.replicate_first_row()
                pipe.filter_and_backproject(out, sht)
                for kk in range(cnt):
                    self.cl_writer.write_data_try(out[kk], params.save_centers[k0 + kk],
                                                  id_slice)
        torch.cuda.synchronize(dev)

    # ------------------------------------------------------------------ device
    def recon_device(self, data, dark0, flat0, out, stream=None):
        """All-device reconstruction: data [nproj, nz, n] (any frame dtype, on device),
        dark0/flat0 [nz, n] resident statistics, out [nz, n, n] float32."""
        ncz, nz = params.ncz, params.nz
        for k in range(params.nzchunk):
            z0 = k * ncz
            lz = int(params.lzchunk[k])
            if lz == ncz:
                self.pipe.reconstruct(out[z0:z0 + ncz], data[:, z0:z0 + ncz], dark0, flat0,
                                      z_lo=z0, stream=stream)
            else:
                tmp = torch.empty((ncz, params.n, params.n), dtype=out.dtype,
                                  device=out.device)
                self.pipe.reconstruct(tmp, data[:, z0:z0 + lz], dark0, flat0, z_lo=z0,
                                      stream=stream)
                out[z0:z0 + lz].copy_(tmp[:lz])
        return out
