"""Device-resident reconstruction of one chunk of sinogram rows.

``SinoPipeline`` is the fused form of the reference's per-chunk sequence
(GPURec.recon_all, src/tomocupy/rec.py:161-179):

    proc_sino/proc_proj  ->  swapaxes  ->  fbp_filter_center  ->  backprojection

executed as native kernels on one stream:

 1. ``tcb_prep_rows``: uint16 frames -> dark/flat -> -log -> sinogram order
    (one pass, no temporaries, no separate transpose copy);
 2. ``tcb_fftfilter_apply`` (widths up to 4096): edge pad + filter + centre
    shift + crop as one length-2n convolution in shared memory, two slices
    per complex transform, written as FourierRec's packed pairs -- for
    power-of-two widths already through the projection FFT -- or as the
    cropped rows of linerec/lprec;
 3. fourierrec: ``tcb_fourierrec_backprojection_slices`` (gridding, 2D FFT,
    deapodization, unpacking into the output slices); linerec/lprec on the
    filtered rows.

Wider rows take the reference's own route: prep into edge-padded rows of
length ne = 4n, ``tcb_filter_apply`` (R2C -> per-slice spectrum -> C2R),
then ``tcb_fourierrec_pack`` (crop + complex pairing) or a crop copy.

``precision="mixed"`` grids fourierrec on the tensor cores
(``TCB_GRID_TENSOR``: fp16 weights and hi/lo values, fp32 accumulation).
Its filter is the fused fp32 filter (``mixed_filter="fft"``, the default:
O(n log n) and faster at every supported width) or, with
``mixed_filter="tensor"``, ``tcb_prep_rows_split16`` (the prep chain written
as fp16 hi/lo planes) followed by the tensor-core filter
``tcb_tcfilter_apply`` (edge pad + filter + centre shift + crop as one
split-precision fp16 GEMM of 3 * 2 n^2 flops per row), whose epilogue writes
the packed complex pairs of fourierrec or the cropped rows of linerec/lprec.
Neither filter modifies its input.
"""
from __future__ import annotations

import math
import os

import numpy as np
import torch

from . import _lib, cfunc_filter, cfunc_fourierrec, cfunc_linerec
from .processing.proc_functions import dezinger as _dezinger
from .processing.proc_functions import in_dtype_code, prep_rows, prep_rows_split16
from .reconstruction.backproj_functions import phase_weights, rfftfreq32
from .reconstruction import fftfilter as _fff
from .reconstruction.fbp_filter import calc_filter


class SinoPipeline:
    def __init__(self, n, nproj, ncz, theta, center, fbp_filter="parzen",
                 algorithm="fourierrec", minus_log=True, device="cuda", stripe=None,
                 precision="float32", out_dtype="float32", mixed_filter="fft", dezinger=None,
                 ni=None, pad360=None, gridding="auto"):
        if algorithm not in ("fourierrec", "linerec", "lprec"):
            raise NotImplementedError(f"SinoPipeline: algorithm {algorithm!r}")
        if precision not in ("float32", "mixed"):
            raise NotImplementedError(f"SinoPipeline: precision {precision!r}")
        self.precision = precision
        if mixed_filter not in ("fft", "tensor"):
            raise NotImplementedError(f"SinoPipeline: mixed_filter {mixed_filter!r}")
        if out_dtype not in ("float32", "float16"):
            raise NotImplementedError(f"SinoPipeline: out_dtype {out_dtype!r}")
        self.out_dtype = torch.float16 if out_dtype == "float16" else torch.float32
        if algorithm == "fourierrec" and ncz % 2:
            raise ValueError("fourierrec needs an even number of rows per chunk")
        self.device = torch.device(device)
        self.n, self.nproj, self.ncz = int(n), int(nproj), int(ncz)
        # lprec reconstructs about centre + 0.5, as BackprojFunctions sets it
        # (reconstruction/backproj_functions.py:70-71)
        self.center = float(center) + (0.5 if algorithm == "lprec" else 0.0)
        self.algorithm = algorithm
        self.minus_log = minus_log
        # outlier removal of the frames of each chunk (proc_sino's
        # remove_outliers): (width, threshold) or None; frames go through a
        # chunk-sized scratch stack
        self.dezinger = dezinger
        self._zbuf = None
        # double field of view (proc_proj's pad360 after -log): frames of ni
        # columns reconstructed at n = 2 ni; pad360 = (flip, w)
        self.ni = int(ni) if ni is not None else self.n
        self.pad360 = None
        if pad360 is not None:
            import ctypes as C
            flip, w = bool(pad360[0]), int(pad360[1])
            if self.ni * 2 != self.n or not 1 <= w <= self.ni:
                raise ValueError(f"pad360: n={self.n} must be 2*ni={2 * self.ni}, 1 <= w <= ni")
            v = np.empty(w, dtype=np.float64)
            _lib.call("tcb_pad360_weights", v.ctypes.data_as(C.c_void_p), w)
            self.pad360 = (flip, w, torch.as_tensor(v, device=self.device))
        elif self.ni != self.n:
            raise ValueError("input width differs from n without double-FOV padding")
        self.ne = 4 * self.n
        self.pad = self.ne // 2 - self.n // 2
        self.theta = torch.as_tensor(np.asarray(theta, dtype=np.float32), device=self.device)
        self.wfilter_np = calc_filter(self.ne, fbp_filter)
        self.wfilter = torch.as_tensor(self.wfilter_np, device=self.device)
        self.t = rfftfreq32(self.ne, self.device)
        self._w_cache: dict = {}
        self.fused = _fff.supported(self.n) and (precision == "float32" or
                                                  mixed_filter == "fft")
        # the tensor-core filter on split fp16 planes (mixed precision only)
        self.tensor_filter = precision == "mixed" and not self.fused
        if self.tensor_filter:
            from .reconstruction.tcfilter import TCFilter
            self.npl = -(-self.n // 8) * 8  # fp16 row pitch (16-byte TMA rows)
            self.xhi = torch.empty((self.ncz, self.nproj, self.npl), dtype=torch.float16,
                                   device=self.device)
            self.xlo = torch.empty_like(self.xhi)
            self.tcf = TCFilter(self.n, self.nproj, self.ncz, 1, self.device)
            self.tcf.set_kernels(self.wfilter_np, self.ne, self.center, 0.0)
            self.tcf_sht = None      # per-slice kernels for centre shifts (built on demand)
            self._sht_key = None
        elif _fff.supported(self.n):
            # fused filter: compact rows, not modified by filtering
            self.rows = torch.empty((self.ncz, self.nproj, self.n), dtype=torch.float32,
                                    device=self.device)
            self.fff = _fff.FFTFilter(self.n, self.nproj, self.ncz, 1, self.device)
            self.fff.set_kernels(self.wfilter_np, self.ne, self.center, 0.0)
            self.fff_sht = None      # per-slice kernels for centre shifts (built on demand)
            self._fff_key = None
        else:
            self.rows = torch.empty((self.ncz, self.nproj, self.ne), dtype=torch.float32,
                                    device=self.device)
            self.filter = cfunc_filter.cfunc_filter(self.nproj, self.ncz, self.ne)
        # optional ring removal between dark/flat and -log (ProcFunctions.proc_sino,
        # proc_functions.py:140-160): stripe is ("ti", beta, mask_size) for
        # Titarenko's method, ("vo-all", snr, la_size, sm_size, dim) for Vo's
        # method, else (sigma, wavelet, level) for the Fourier-wavelet method;
        # all work in place on sinograms in self.sino
        self.fw = None
        if stripe is not None and stripe[0] == "ti":
            from .processing.remove_stripe import StripeTI
            self.fw = StripeTI(self.nproj, self.ncz, self.ni, stripe[1], stripe[2])
        elif stripe is not None and stripe[0] == "vo-all":
            from .processing.remove_stripe import StripeVO
            self.fw = StripeVO(self.nproj, self.ncz, self.ni, *stripe[1:])
        elif stripe is not None:
            from .processing.remove_stripe import StripeFW
            sigma, wname, level = stripe
            self.fw = StripeFW(self.nproj, self.ncz, self.ni, sigma, wname, level)
        if self.fw is not None:
            # ni-wide sinograms: double-FOV scans are padded after ring removal
            self.sino = torch.zeros((self.ncz, self.fw.nproj_pad, self.ni), dtype=torch.float32,
                                    device=self.device)
        if algorithm == "fourierrec":
            self.fr = cfunc_fourierrec.cfunc_fourierrec(self.nproj, self.ncz // 2, self.n,
                                                        self.theta)
            self.gridding = self._set_gridding(gridding, precision)
            if out_dtype == "float16":
                self.fr.set_output(_lib.TCB_FLOAT16)
            # the fused filter hands over the projection FFT already done
            self.fr_spectrum = self.fused and _fff.spectrum_supported(self.n)
            if self.fr_spectrum:
                self.fr.set_input_spectrum(True)
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
            # fp16 output slices (the reference's float16 path returns fp16
            # volumes): lprec and linerec accumulate in fp32 here, then round
            self.out32 = (torch.empty((self.ncz, self.n, self.n), dtype=torch.float32,
                                      device=self.device)
                          if self.out_dtype == torch.float16 else None)

    def _set_gridding(self, gridding: str, precision: str) -> int:
        """fourierrec gridding mode.  'auto': the tensor cores with streamed
        weights (split fp16 for float32, fp16 for mixed) when their tables fit
        in device memory, else the fp32 register gridding (float32) or the
        tensor-core gridding that builds its weights per chunk (mixed).
        'fp32' / 'tensor' / 'tensor_fp32' / 'tensor_stream' force a mode."""
        modes = {"fp32": _lib.GRID_FP32, "tensor": _lib.GRID_TENSOR,
                 "tensor_fp32": _lib.GRID_TENSOR_FP32, "tensor_stream": _lib.GRID_TENSOR_STREAM}
        if gridding != "auto":
            self.fr.set_gridding(modes[gridding])
            return modes[gridding]
        first = _lib.GRID_TENSOR_STREAM if precision == "mixed" else _lib.GRID_TENSOR_FP32
        if os.environ.get("TCB_FOURIERREC_GRIDDING") in modes:
            first = modes[os.environ["TCB_FOURIERREC_GRIDDING"]]
        fallback = _lib.GRID_TENSOR if precision == "mixed" else _lib.GRID_FP32
        try:
            self.fr.set_gridding(first)
            return first
        except _lib.TcbError as e:
            if e.status != _lib.TCB_ERR_OUT_OF_MEMORY:
                raise
        self.fr.set_gridding(fallback)
        return fallback

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

    def load_rows(self, data, dark0=None, flat0=None, z_lo=0, stream=None, flat1=None,
                  row0=0):
        """Fill the padded filter rows from a [nproj, nz, n] frame (or float) stack view.
        flat1: the second flat mean of flat_linear (the per-angle blend of
        proc_functions.py:62-66), or None.  row0: first filter row to fill
        (several stacks packed into one chunk; plain fused pipelines only)."""
        nz = data.shape[1]
        assert row0 + nz <= self.ncz and data.shape[0] == self.nproj and data.shape[2] == self.ni
        if row0:
            if (self.dezinger is not None or self.fw is not None or self.tensor_filter
                    or not self.fused or self.pad360 is not None):
                raise NotImplementedError("rows packed at an offset: plain fused pipelines only")
            prep_rows(self.rows[row0:], data, None if dark0 is None else dark0[z_lo:z_lo + nz],
                      None if flat0 is None else flat0[z_lo:z_lo + nz],
                      None if flat1 is None else flat1[z_lo:z_lo + nz],
                      darkflat=dark0 is not None, minus_log=self.minus_log,
                      flat_linear=flat1 is not None, out_zstride=self.nproj * self.n,
                      out_pstride=self.n, stream=stream)
            return
        if self.pad360 is not None and not self.fused:
            raise NotImplementedError("double-FOV padding: fused fp32 filter only")
        if self.dezinger is not None:
            if self._zbuf is None or self._zbuf.dtype != data.dtype:
                self._zbuf = torch.empty((self.nproj, self.ncz, self.ni), dtype=data.dtype,
                                         device=self.device)
            # a contiguous [nproj, nz, n] view of the scratch (partial chunks too)
            # frames arrive at the input width ni (double-FOV scans reconstruct at n = 2 ni)
            zb = self._zbuf.view(-1)[:self.nproj * nz * self.ni].view(self.nproj, nz, self.ni)
            data = _dezinger(data, *self.dezinger, out=zb, stream=stream)
        d0 = dark0[z_lo:z_lo + nz] if dark0 is not None else None
        f0 = flat0[z_lo:z_lo + nz] if flat0 is not None else None
        f1 = flat1[z_lo:z_lo + nz] if flat1 is not None else None
        fl = dict(flat1=f1, flat_linear=f1 is not None)
        if self.fw is not None:
            fw = self.fw
            s = torch.cuda.current_stream() if stream is None else stream
            with torch.cuda.stream(s) if not isinstance(s, int) else _nullctx():
                self.sino.zero_()
            prep_rows(self.sino, data, d0, f0, darkflat=dark0 is not None, minus_log=False,
                      out_zstride=fw.nproj_pad * self.ni, out_pstride=self.ni,
                      out_poff=fw.poff, stream=stream, **fl)
            fw.apply_sino(self.sino, stream)
            src = self.sino[:nz, fw.poff:fw.poff + self.nproj].permute(1, 0, 2)
            if self.tensor_filter:
                prep_rows_split16(self.xhi, self.xlo, src, darkflat=False,
                                  minus_log=self.minus_log, out_zstride=self.nproj * self.npl,
                                  out_pstride=self.npl, stream=stream)
                return
            if self.fused:
                prep_rows(self.rows, src, darkflat=False, minus_log=self.minus_log,
                          out_zstride=self.nproj * self.n, out_pstride=self.n, stream=stream)
                self._pad360_rows(nz, stream)
                return
            prep_rows(self.rows, src, darkflat=False, minus_log=self.minus_log,
                      out_zstride=self.nproj * self.ne, out_pstride=self.ne, out_xoff=self.pad,
                      out_width=self.ne, edge_pad=True, stream=stream)
            return
        if self.tensor_filter:
            prep_rows_split16(self.xhi, self.xlo, data, d0, f0, darkflat=dark0 is not None,
                              minus_log=self.minus_log, out_zstride=self.nproj * self.npl,
                              out_pstride=self.npl, stream=stream, **fl)
            return
        if self.fused:
            prep_rows(self.rows, data, d0, f0, darkflat=dark0 is not None,
                      minus_log=self.minus_log, out_zstride=self.nproj * self.n,
                      out_pstride=self.n, stream=stream, **fl)
            self._pad360_rows(nz, stream)
            return
        prep_rows(self.rows, data, d0, f0, darkflat=dark0 is not None,
                  minus_log=self.minus_log, out_zstride=self.nproj * self.ne,
                  out_pstride=self.ne, out_xoff=self.pad, out_width=self.ne, edge_pad=True,
                  stream=stream, **fl)

    def _pad360_rows(self, nz: int, stream=None) -> None:
        """Double-FOV padding of the -log rows of nz slices, in place (ni -> 2 ni)."""
        if self.pad360 is None:
            return
        flip, w, v = self.pad360
        _lib.call("tcb_pad360_rows", self.rows.data_ptr(), nz * self.nproj, self.ni,
                  self.n, int(flip), v.data_ptr(), w, _lib.stream_ptr(stream))

    def clear_rows(self, lz: int, stream=None) -> None:
        """Zero the filter input rows of slices [lz, ncz) (a partial chunk).

        fourierrec pairs slice k with slice k + ncz/2, so leftover rows of an
        earlier chunk would leak into a partial chunk through the packing's
        real/imaginary crosstalk; zero rows make every chunk depend on its own
        slices only.
        """
        if lz >= self.ncz:
            return
        s = torch.cuda.current_stream() if stream is None else stream
        with torch.cuda.stream(s) if not isinstance(s, int) else _nullctx():
            if self.tensor_filter:
                self.xhi[lz:].zero_()
                self.xlo[lz:].zero_()
            else:
                self.rows[lz:].zero_()

    def replicate_first_row(self):
        """Copy slice 0 of the loaded rows to every slice (try-centre sweeps)."""
        if self.tensor_filter:
            self.xhi[1:].copy_(self.xhi[:1].expand(self.ncz - 1, -1, -1))
            self.xlo[1:].copy_(self.xlo[:1].expand(self.ncz - 1, -1, -1))
        else:
            self.rows[1:].copy_(self.rows[:1].expand(self.ncz - 1, -1, -1))

    def save_rows(self):
        """Snapshot of slice 0 needed to refill rows that filtering overwrote (or None)."""
        return None if (self.tensor_filter or self.fused) else self.rows[0].clone()

    def restore_rows(self, saved):
        if saved is not None:
            self.rows.copy_(saved.expand(self.ncz, -1, -1))

    def _tc_filter(self, sht):
        """The tensor-core filter for these centre shifts (shared kernel when None)."""
        if sht is None:
            return self.tcf
        from .reconstruction.tcfilter import TCFilter
        sh = np.asarray(sht, dtype=np.float32).reshape(-1)
        if sh.size == 1:
            sh = np.repeat(sh, self.ncz)
        if self.tcf_sht is None:
            self.tcf_sht = TCFilter(self.n, self.nproj, self.ncz, self.ncz, self.device)
        key = sh.tobytes()
        if key != self._sht_key:
            self.tcf_sht.set_kernels(self.wfilter_np, self.ne, self.center, sh.astype(np.float64))
            self._sht_key = key
        return self.tcf_sht

    def _fft_filter(self, sht):
        """The fused filter for these centre shifts (shared kernel when None)."""
        if sht is None:
            return self.fff
        sh = np.asarray(sht, dtype=np.float32).reshape(-1)
        if sh.size == 1:
            sh = np.repeat(sh, self.ncz)
        if self.fff_sht is None:
            self.fff_sht = _fff.FFTFilter(self.n, self.nproj, self.ncz, self.ncz, self.device)
        key = sh.tobytes()
        if key != self._fff_key:
            self.fff_sht.set_kernels(self.wfilter_np, self.ne, self.center,
                                     sh.astype(np.float64))
            self._fff_key = key
        return self.fff_sht

    def _filter_and_backproject_fused(self, out, sht, stream, kern0=0, fff=None):
        f = fff if fff is not None else self._fft_filter(sht)
        if self.algorithm == "fourierrec":
            f.apply(self.rows, torch.view_as_complex(self.g),
                    "spectrum" if self.fr_spectrum else "pairs", kern0=kern0, stream=stream)
            self.fr.backprojection_slices(out, self.g, stream)
            return out
        f.apply(self.rows, self.crop, "rows", kern0=kern0, stream=stream)
        if self.algorithm == "linerec":
            s = torch.cuda.current_stream() if stream is None else stream
            with torch.cuda.stream(s) if not isinstance(s, int) else _nullctx():
                out.zero_()
            self.lr.backprojection(out, self.crop, self.theta, math.pi / 2, 0, stream)
        else:
            self.lp.fslv.backprojection(out, self.crop, stream)
        return out

    def _filter_and_backproject_mixed(self, out, sht, stream):
        f = self._tc_filter(sht)
        if self.algorithm == "fourierrec":
            f.apply(self.xhi, self.xlo, torch.view_as_complex(self.g), pairs=True, stream=stream)
            self.fr.backprojection_slices(out, self.g, stream)
            return out
        f.apply(self.xhi, self.xlo, self.crop, stream=stream)
        if self.algorithm == "linerec":
            s = torch.cuda.current_stream() if stream is None else stream
            with torch.cuda.stream(s) if not isinstance(s, int) else _nullctx():
                out.zero_()
            self.lr.backprojection(out, self.crop, self.theta, math.pi / 2, 0, stream)
        else:
            self.lp.fslv.backprojection(out, self.crop, stream)
        return out

    def filter_and_backproject(self, out, sht=None, stream=None):
        """out [ncz, n, n] of self.out_dtype (contiguous) from the loaded rows."""
        assert out.dtype == self.out_dtype, (out.dtype, self.out_dtype)
        if self.algorithm != "fourierrec" and out.dtype == torch.float16:
            self._filter_and_backproject32(self.out32[:out.shape[0]], sht, stream)
            s = torch.cuda.current_stream() if stream is None else stream
            with torch.cuda.stream(s) if not isinstance(s, int) else _nullctx():
                out.copy_(self.out32[:out.shape[0]])
            return out
        return self._filter_and_backproject32(out, sht, stream)

    def _filter_and_backproject32(self, out, sht=None, stream=None):
        if self.tensor_filter:
            return self._filter_and_backproject_mixed(out, sht, stream)
        if self.fused:
            return self._filter_and_backproject_fused(out, sht, stream)
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

    def reconstruct(self, out, data, dark0=None, flat0=None, z_lo=0, sht=None, stream=None,
                    flat1=None):
        self.load_rows(data, dark0, flat0, z_lo, stream, flat1=flat1)
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
    if src.stride(1) != c or dst.stride(1) != c:
        # rows narrower than their pitch (a column range of the frames, e.g.
        # the float16 power-of-two crop): one 2D copy of b rows per a
        for i in range(a):
            _lib.call("tcb_copy2d", dst[i].data_ptr(), dst.stride(1) * es, src[i].data_ptr(),
                      src.stride(1) * es, c * es, b, _lib.stream_ptr(stream))
        return
    _lib.call("tcb_copy2d", dst.data_ptr(), dst.stride(0) * es, src.data_ptr(),
              src.stride(0) * es, b * c * es, a, _lib.stream_ptr(stream))
