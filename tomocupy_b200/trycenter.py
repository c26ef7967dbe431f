"""Try-centre sweeps: every centre of a rotation-axis search in one CUDA graph.

The reference reconstructs one slice for a list of candidate rotation
centres by tiling the slice ``ncz`` times, filtering each copy with its own
centre shift and running one fourierrec launch per chunk, with host
synchronisation per chunk (GPURec.recon_try, src/tomocupy/rec.py:210-275;
Reader.init_sizes_try, src/tomocupy/dataio/reader.py:224-247).

``TryCenterSweep`` keeps everything of a sweep resident -- the normalised
slice, per-centre filter operators (the tensor-core Toeplitz operators in
mixed precision, the fused filter's per-centre convolution spectra in fp32),
the gridding tables and the output stack of all centres -- and records the
whole sweep (filter -> 1D FFT -> gridding -> pruned 2D FFT -> deapodization
for every chunk) into one CUDA graph.  A sweep is then one graph launch.  ``autotune`` times the
sweep for each candidate chunk size and gridding depth (slice pairs per
gridding block) on the actual geometry and keeps the fastest.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import torch

from .pipeline import SinoPipeline


def chunk_shifts(shifts, ncz: int) -> np.ndarray:
    """float32 [nchunks, ncz] centre shifts, zero-padded past the last centre."""
    sh = np.asarray(shifts, dtype=np.float32).reshape(-1)
    nch = max(1, math.ceil(sh.size / ncz))
    out = np.zeros((nch, ncz), dtype=np.float32)
    out.reshape(-1)[:sh.size] = sh
    return out


def per_center_errors(a: torch.Tensor, b: torch.Tensor):
    """(rel-L2, max-abs) per centre of two [S, n, n] stacks (float64 on the host)."""
    rel, mx = [], []
    for k in range(a.shape[0]):
        d = (a[k].double() - b[k].double())
        rel.append(float(torch.linalg.vector_norm(d) /
                         torch.linalg.vector_norm(b[k].double()).clamp_min(1e-300)))
        mx.append(float(d.abs().max()))
    return np.array(rel), np.array(mx)


class TryCenterSweep:
    """One slice reconstructed for ``len(shifts)`` centre shifts (fourierrec).

    shifts are relative to ``center`` with the sign of the reference's
    ``sht`` (the filter shifts the rotation axis to ``center - sht``).
    """

    def __init__(self, n, nproj, theta, center, shifts, fbp_filter="parzen",
                 precision="float32", ncz=32, pairs_per_block=0, device="cuda",
                 minus_log=True, mixed_filter="fft", ni=None, pad360=None, stripe=None):
        self.device = torch.device(device)
        self.n, self.nproj, self.ncz = int(n), int(nproj), int(ncz)
        self.precision = precision
        self.shifts = np.asarray(shifts, dtype=np.float32).reshape(-1)
        self.S = self.shifts.size
        self.sht = chunk_shifts(self.shifts, self.ncz)
        self.nchunks = self.sht.shape[0]
        # ni / pad360: a double-FOV scan (frames of ni columns, pad360 after -log);
        # stripe: ring removal of the slice (SinoPipeline's stripe argument)
        self.pipe = SinoPipeline(self.n, self.nproj, self.ncz, theta, center, fbp_filter,
                                 "fourierrec", minus_log=minus_log, device=self.device,
                                 stripe=stripe, precision=precision, mixed_filter=mixed_filter,
                                 ni=ni, pad360=pad360)
        if pairs_per_block:
            self.pipe.fr.set_pairs_per_block(pairs_per_block)
        self.pairs_per_block = int(pairs_per_block)
        self.out = torch.empty((self.nchunks * self.ncz, self.n, self.n), dtype=torch.float32,
                               device=self.device)
        if self.pipe.tensor_filter:
            from .reconstruction.tcfilter import TCFilter
            self.tcf = TCFilter(self.n, self.nproj, self.ncz, self.nchunks * self.ncz,
                                self.device)
            self.tcf.set_kernels(self.pipe.wfilter_np, self.pipe.ne, self.pipe.center,
                                 self.sht.reshape(-1).astype(np.float64))
        elif self.pipe.fused:
            from .reconstruction.fftfilter import FFTFilter
            self.fff = FFTFilter(self.n, self.nproj, self.ncz, self.nchunks * self.ncz,
                                 self.device)
            self.fff.set_kernels(self.pipe.wfilter_np, self.pipe.ne, self.pipe.center,
                                 self.sht.reshape(-1).astype(np.float64))
        else:
            self.weights = [self.pipe.weights(self.sht[k]) for k in range(self.nchunks)]
        self.saved = None
        self.graph = None
        self._stream = torch.cuda.Stream(self.device)

    # ------------------------------------------------------------------ data
    def load(self, data, dark0=None, flat0=None, flat1=None):
        """Normalise one slice of frames (data [nproj, 1, n] on the device) into the
        rows (flat1: the second flat mean of flat_linear, or None)."""
        with torch.cuda.stream(self._stream):
            self.pipe.load_rows(data, dark0, flat0, 0, self._stream, flat1=flat1)
            self.pipe.replicate_first_row()
            if not self.pipe.tensor_filter and not self.pipe.fused:
                # same buffer on every load: a captured graph reads it
                if self.saved is None:
                    self.saved = self.pipe.rows[0].clone()
                else:
                    self.saved.copy_(self.pipe.rows[0])
        self._stream.synchronize()

    # ------------------------------------------------------------------ work
    def _enqueue(self, stream):
        p = self.pipe
        for k in range(self.nchunks):
            outk = self.out[k * self.ncz:(k + 1) * self.ncz]
            if p.tensor_filter:
                self.tcf.apply(p.xhi, p.xlo, torch.view_as_complex(p.g), pairs=True,
                               kern0=k * self.ncz, stream=stream)
            elif p.fused:  # the fused filter leaves the rows as they are
                self.fff.apply(p.rows, torch.view_as_complex(p.g),
                               "spectrum" if p.fr_spectrum else "pairs", kern0=k * self.ncz,
                               stream=stream)
            else:
                # the cuFFT filter works in place: refill the rows of every chunk
                p.rows.copy_(self.saved.expand(self.ncz, -1, -1))
                p.filter.filter(p.rows, self.weights[k], stream)
                p.fr.pack(p.g, p.rows, p.ne, p.pad, stream)
            p.fr.backprojection_slices(outk, p.g, stream)

    def capture(self) -> None:
        """Record the whole sweep into one CUDA graph (after a warm-up run)."""
        s = self._stream
        with torch.cuda.stream(s):
            self._enqueue(s)  # warm-up: plans, lazy module loading
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self._enqueue(s)
        s.synchronize()
        self.graph = g

    def run(self) -> torch.Tensor:
        """Reconstruct every centre; returns the [S, n, n] view of the output stack."""
        s = self._stream
        if self.graph is not None:
            with torch.cuda.stream(s):
                self.graph.replay()
        else:
            with torch.cuda.stream(s):
                self._enqueue(s)
        s.synchronize()
        return self.out[:self.S]

    def time_ms(self, reps=3) -> float:
        """Device time of one sweep (graph replay when captured), CUDA events."""
        s = self._stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            e0.record(s)
            for _ in range(reps):
                if self.graph is not None:
                    self.graph.replay()
                else:
                    self._enqueue(s)
            e1.record(s)
        s.synchronize()
        return e0.elapsed_time(e1) / reps

    def free(self):
        self.graph = None
        for name in ("tcf", "fff"):
            obj = getattr(self, name, None)
            if obj is not None:
                obj.free()
        self.pipe = None
        self.out = None


# ---------------------------------------------------------------------- tuning
_TUNED: dict = {}


def autotune(n, nproj, theta, center, shifts, data, dark0=None, flat0=None, *,
             fbp_filter="parzen", precision="float32", candidates=None, reps=2,
             cache_file=None, device="cuda"):
    """Pick (ncz, pairs_per_block) with the fastest captured sweep for this geometry.

    candidates: iterable of (ncz, pairs_per_block); by default chunk sizes
    32..128 when the geometry's gridding runs on the tensor cores with
    streamed weights (pairs_per_block does not apply there), else chunk sizes
    8..64 with register-gridding depths 4..16 pairs.  Returns {"ncz",
    "pairs_per_block", "ms", "table"}; results are cached per geometry
    in-process and, when cache_file is given, in that JSON file.
    """
    key = f"{n}x{nproj}x{len(np.atleast_1d(shifts))}:{precision}:{fbp_filter}"
    if key in _TUNED:
        return _TUNED[key]
    if cache_file is not None and Path(cache_file).exists():
        saved = json.loads(Path(cache_file).read_text())
        if key in saved:
            _TUNED[key] = saved[key]
            return saved[key]
    first = None
    if candidates is None:
        first = TryCenterSweep(n, nproj, theta, center, shifts, fbp_filter, precision, 64, 0,
                               device)
        from . import _lib
        if first.pipe.gridding in (_lib.GRID_TENSOR_FP32, _lib.GRID_TENSOR_STREAM):
            candidates = [(64, 0), (32, 0), (128, 0)]
        else:
            candidates = [(ncz, zb) for ncz in (8, 16, 32, 64) for zb in (4, 8, 16)
                          if zb <= ncz // 2]
            first.free()
            first = None
    table = []
    for ncz, zb in candidates:
        if first is not None and (ncz, zb) == (64, 0):
            sw, first = first, None
        else:
            sw = TryCenterSweep(n, nproj, theta, center, shifts, fbp_filter, precision, ncz, zb,
                                device)
        sw.load(data, dark0, flat0)
        sw.capture()
        sw.time_ms(1)
        ms = sw.time_ms(reps)
        table.append({"ncz": ncz, "pairs_per_block": zb, "ms": round(ms, 3)})
        sw.free()
        del sw
        torch.cuda.empty_cache()
    best = min(table, key=lambda r: r["ms"])
    res = {"ncz": best["ncz"], "pairs_per_block": best["pairs_per_block"], "ms": best["ms"],
           "table": table}
    _TUNED[key] = res
    if cache_file is not None:
        p = Path(cache_file)
        saved = json.loads(p.read_text()) if p.exists() else {}
        saved[key] = res
        p.write_text(json.dumps(saved, indent=1))
    return res
