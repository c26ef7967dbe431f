"""Reconstruction serving: continuous batching of uneven requests on one GPU.

A request is one tomographic reconstruction (uint16 frames [nproj, nz, n],
darks, flats, angles, centre, precision).  The server keeps per-geometry
state resident -- the chunk pipeline with its filter spectra or tensor-core
filter operators, the gridding sample lists and deapodization constants --
and per-request dark/flat statistics, and runs a continuous-batching loop:

* admission: a request that has arrived is admitted when its device bytes
  (frames, darks, flats, statistics) plus the resident geometries fit the HBM
  budget; its frames go to the device on a copy stream;
* dispatch: every geometry stream with room takes the next ``ncz`` slices of
  its oldest admitted request and, for mixed-precision requests, when that
  request has fewer left, fills the rest of the chunk with the next slices
  of the other admitted requests of the same geometry (their frames are
  normalised into the chunk's rows side by side, then one filter, gridding
  and inverse-FFT launch serves them all); requests of different widths,
  angle counts and slice counts run concurrently on their own streams, and
  a request that arrives while others run starts as soon as a stream has
  room;
* completion: each chunk's slices are copied back to the request's pinned
  host output on the slot's stream; a request is done when its last chunk's
  copy is.

Partial chunks are zero-filled.  fourierrec packs slice k of a chunk with
slice k + ncz/2 as the real and imaginary parts of one complex sinogram
(the reference's FourierRec does the same), and the polar samples are not
symmetric about the origin (radii -n/2 .. n/2 - 1), so a slice's result
carries ~1e-4 (relative) of its partner's: a slice paired with another
request's slice differs from the same slice paired with zeros by that much.
fp32 requests are therefore never packed with others (every chunk holds one
request's slices: bit-identical alone and in any mix, and paired as
GPURec pairs them); mixed-precision requests, whose budget is 1e-3, are
(tested within 1e-3 of alone).

The reference has no serving layer; the per-request computation is the same
as GPURec.recon_all (src/tomocupy/rec.py:113-208).
"""
from __future__ import annotations

import time
from collections import OrderedDict
from dataclasses import dataclass, field

import numpy as np
import torch

from .pipeline import SinoPipeline, copy2d_rows
from .processing.proc_functions import darkflat_stats


@dataclass
class Request:
    """One reconstruction.  frames/dark/flat are host tensors (pinned for async copies)."""
    rid: int
    frames: torch.Tensor          # uint16 [nproj, nz, n]
    dark: torch.Tensor            # [ndark, nz, n]
    flat: torch.Tensor            # [nflat, nz, n]
    theta: np.ndarray             # float32 [nproj]
    center: float
    precision: str = "float32"    # "float32" | "mixed"
    fbp_filter: str = "parzen"
    arrival: float = 0.0          # seconds after the start of the stream
    out: torch.Tensor | None = None   # pinned host [nz, n, n] (given or allocated)
    out_dtype: str = "float32"    # "float16": fp16 slices (half the result bytes)
    # filled in by the server
    t_admit: float = float("nan")
    t_done: float = float("nan")

    @property
    def shape(self):
        return tuple(self.frames.shape)

    @property
    def gups_work(self) -> float:
        nproj, nz, n = self.frames.shape
        return float(n) * n * nz * nproj

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def _geometry_key(req: Request, ncz: int):
    nproj, _, n = req.frames.shape
    th = np.asarray(req.theta, dtype=np.float32)
    return (n, nproj, hash(th.tobytes()), float(req.center), req.fbp_filter, req.precision,
            req.out_dtype, ncz)


@dataclass
class _Geometry:
    pipe: SinoPipeline     # resident tables, spectra / operators, scratch
    tmp: list              # two [ncz, n, n] float32 output staging buffers
    stream: torch.cuda.Stream   # chunks of this geometry run in order on it
    d2h: torch.cuda.Stream      # result copies, off the compute stream
    nbytes: int = 0
    users: int = 0         # admitted requests using it
    inflight: list = field(default_factory=list)   # compute events of queued chunks
    tmp_free: list = field(default_factory=lambda: [None, None])  # copy-out done events
    flip: int = 0


@dataclass
class _Active:
    req: Request
    key: tuple
    frames: torch.Tensor
    dark0: torch.Tensor
    flat0: torch.Tensor
    ready: torch.cuda.Event
    nz: int
    nbytes: int
    z_next: int = 0        # first slice not yet dispatched
    events: list = field(default_factory=list)

    @property
    def pending(self) -> bool:
        return self.z_next < self.nz


class Server:
    """Continuous-batching reconstruction server on one GPU.

    hbm_budget: bytes of device memory the server may hold (resident
    geometries + admitted requests).  ncz: slices per chunk.  depth: chunks
    queued ahead per geometry stream.  max_active: admitted requests at most
    (None = memory-bound only; 1 gives one-at-a-time serving).  pack: fill
    a chunk with the slices of several mixed-precision requests of one
    geometry.
    """

    def __init__(self, device="cuda", hbm_budget=150e9, ncz=8, depth=2, max_active=None,
                 pack=True):
        self.device = torch.device(device)
        self.budget = float(hbm_budget)
        self.ncz = int(ncz)
        self.depth = int(depth)
        self.max_active = max_active
        self.pack = bool(pack)
        self.chunks = 0           # chunk launches (last serve call)
        self.copy_stream = torch.cuda.Stream(self.device)
        self.d2h = torch.cuda.Stream(self.device)
        self.geoms: OrderedDict = OrderedDict()
        self.geom_bytes = 0
        self.req_bytes = 0
        self.peak_active = 0      # most requests admitted at once (last serve call)
        self.peak_bytes = 0       # most budgeted bytes held at once (last serve call)

    # ------------------------------------------------------------ geometry
    def _free_dev(self) -> int:
        return torch.cuda.mem_get_info(self.device)[0]

    def geometry(self, req: Request) -> _Geometry:
        """Resident state for the request's geometry (built on first use, LRU)."""
        key = _geometry_key(req, self.ncz)
        g = self.geoms.get(key)
        if g is not None:
            self.geoms.move_to_end(key)
            return g
        nproj, _, n = req.frames.shape
        est = self._estimate_geometry_bytes(n, nproj, req.precision)
        self._evict(est)
        torch.cuda.synchronize(self.device)
        before = self._free_dev()
        pipe = SinoPipeline(n, nproj, self.ncz, req.theta, req.center, req.fbp_filter,
                            "fourierrec", device=self.device, precision=req.precision,
                            out_dtype=req.out_dtype,
                            # per-chunk weights: no per-geometry weight tables
                            # (up to 37 GB for 4096 x 3000) in the resident set
                            gridding="tensor" if req.precision == "mixed" else "fp32")
        tmp = [torch.empty((self.ncz, n, n), dtype=pipe.out_dtype, device=self.device)
               for _ in range(2)]
        torch.cuda.synchronize(self.device)
        nb = max(before - self._free_dev(), 2 * tmp[0].numel() * tmp[0].element_size())
        # one copy-out stream for every geometry: results cross the host link
        # one at a time in dispatch (oldest-request-first) order, the order
        # that keeps the longest waits shortest on a shared link, instead of
        # sharing its bandwidth among all requests in flight
        g = _Geometry(pipe, tmp, torch.cuda.Stream(self.device), self.d2h, nb)
        self.geoms[key] = g
        self.geom_bytes += nb
        return g

    def _estimate_geometry_bytes(self, n, nproj, precision) -> int:
        ncz = self.ncz
        rows = ncz * nproj * n * (4 if n <= 4096 else 16)  # fused filter: unpadded rows
        grid = (ncz // 2) * (2 * n) ** 2 * 8 * 2     # grid + FFT work area
        lists = nproj * n * 4 * 8
        tc = 20 * 4 * 2 * nproj * n if precision == "mixed" else 0  # gridding records
        return rows + grid + lists + tc + 2 * ncz * n * n * 4 + (ncz // 2) * nproj * n * 8

    def _evict(self, need: int) -> None:
        for key in list(self.geoms.keys()):
            if self.geom_bytes + self.req_bytes + need <= self.budget:
                return
            g = self.geoms[key]
            if g.users == 0 and not g.inflight:
                self.geom_bytes -= g.nbytes
                del self.geoms[key]
                del g
                torch.cuda.empty_cache()

    def warm(self, requests) -> None:
        """Build the resident state of every geometry in ``requests`` ahead of time."""
        for r in requests:
            self.geometry(r)
        torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------ requests
    def _request_bytes(self, req: Request) -> int:
        nproj, nz, n = req.frames.shape
        return (req.frames.numel() * req.frames.element_size() +
                req.dark.numel() * req.dark.element_size() +
                req.flat.numel() * req.flat.element_size() + 2 * nz * n * 4)

    def _admit(self, req: Request, now: float):
        need = self._request_bytes(req)
        key = _geometry_key(req, self.ncz)
        if key not in self.geoms:
            nproj, _, n = req.frames.shape
            need_g = self._estimate_geometry_bytes(n, nproj, req.precision)
        else:
            need_g = 0
        if self.geom_bytes + self.req_bytes + need + need_g > self.budget:
            self._evict(need + need_g)
            if self.geom_bytes + self.req_bytes + need + need_g > self.budget:
                return None
        g = self.geometry(req)
        nproj, nz, n = req.frames.shape
        cs = self.copy_stream
        with torch.cuda.stream(cs):
            # strided host views (a slab of a larger stack) move with one 2D copy each
            frames, dark, flat = (self._to_device(t, cs) for t in (req.frames, req.dark,
                                                                  req.flat))
            dark0, flat0, _ = darkflat_stats(dark, flat, 1.0, False, cs)
            ready = torch.cuda.Event()
            ready.record(cs)
        if req.out is None:
            req.out = torch.empty((nz, n, n), pin_memory=True,
                                  dtype=torch.float16 if req.out_dtype == "float16"
                                  else torch.float32)
        self.req_bytes += need
        g.users += 1
        req.t_admit = now
        return _Active(req, key, frames, dark0, flat0, ready, nz, need)

    def _to_device(self, t: torch.Tensor, stream) -> torch.Tensor:
        d = torch.empty(tuple(t.shape), dtype=t.dtype, device=self.device)
        if t.stride(2) == 1 and t.stride(1) == t.shape[2]:
            copy2d_rows(d, t, stream)
        else:
            d.copy_(t, non_blocking=True)
        return d

    def _dispatch(self, a: _Active, active: list) -> None:
        """One chunk on a's geometry stream: a's next slices, then (packing)
        the next slices of the other admitted requests of that geometry."""
        g = self.geoms[a.key]
        segs, row = [], 0
        packs = self.pack and a.req.precision == "mixed"
        for b in [a] + ([x for x in active if x is not a and x.key == a.key] if packs
                        else []):
            if row == self.ncz:
                break
            if not b.pending:
                continue
            lz = min(self.ncz - row, b.nz - b.z_next)
            segs.append((b, b.z_next, lz, row))
            b.z_next += lz
            row += lz
        s = g.stream
        i = g.flip
        g.flip ^= 1
        tmp = g.tmp[i]
        for b, _, _, _ in segs:
            s.wait_event(b.ready)
        if g.tmp_free[i] is not None:
            s.wait_event(g.tmp_free[i])  # the previous copy-out of this buffer
        with torch.cuda.stream(s):
            g.pipe.clear_rows(row, s)
            for b, z0, lz, r0 in segs:
                g.pipe.load_rows(b.frames[:, z0:z0 + lz], b.dark0, b.flat0, z_lo=z0, stream=s,
                                 row0=r0)
            g.pipe.filter_and_backproject(tmp, stream=s)
            done = torch.cuda.Event()
            done.record(s)
        self.chunks += 1
        g.d2h.wait_event(done)
        with torch.cuda.stream(g.d2h):
            for b, z0, lz, r0 in segs:
                b.req.out[z0:z0 + lz].copy_(tmp[r0:r0 + lz], non_blocking=True)
            copied = torch.cuda.Event()
            copied.record(g.d2h)
        g.tmp_free[i] = copied
        g.inflight.append(done)
        for b, _, _, _ in segs:
            b.events.append(copied)

    def _finish(self, a: _Active, now: float) -> None:
        a.req.t_done = now
        self.req_bytes -= a.nbytes
        self.geoms[a.key].users -= 1
        a.frames = a.dark0 = a.flat0 = None

    # ------------------------------------------------------------ loop
    def serve(self, requests, realtime=True):
        """Run the stream: requests arrive at their ``arrival`` times (seconds).

        Returns the requests with t_admit/t_done filled and results in .out.
        With realtime=False every request is available at once.
        """
        pending = sorted(requests, key=lambda r: r.arrival)
        active: list[_Active] = []
        self.peak_active = 0
        self.peak_bytes = 0
        self.chunks = 0
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            progressed = False
            # admission, in arrival order
            while pending and (not realtime or pending[0].arrival <= now):
                if self.max_active is not None and len(active) >= self.max_active:
                    break
                a = self._admit(pending[0], now)
                if a is None:
                    break
                pending.pop(0)
                active.append(a)
                self.peak_active = max(self.peak_active, len(active))
                self.peak_bytes = max(self.peak_bytes, self.geom_bytes + self.req_bytes)
                progressed = True
            # retire finished chunks per geometry stream
            for g in self.geoms.values():
                while g.inflight and g.inflight[0].query():
                    g.inflight.pop(0)
            # dispatch, oldest admitted request first: each request gets chunks
            # while its geometry stream has room; requests of other geometries
            # fill their own streams, so everything admitted runs concurrently
            for a in active:
                g = self.geoms[a.key]
                while a.pending and len(g.inflight) < self.depth:
                    self._dispatch(a, active)
                    progressed = True
            # completion
            for a in list(active):
                if not a.pending and all(e.query() for e in a.events):
                    self._finish(a, time.perf_counter() - t0)
                    active.remove(a)
                    progressed = True
            if not progressed:
                time.sleep(2e-5)
        torch.cuda.synchronize(self.device)
        return requests


def latency_summary(requests) -> dict:
    lat = np.array([r.latency for r in requests]) * 1e3
    work = sum(r.gups_work for r in requests)
    span = max(r.t_done for r in requests) - min(r.arrival for r in requests)
    return {"requests": len(requests), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "max_ms": float(lat.max()), "makespan_s": float(span),
            "GUPS": float(work / span / 1e9)}


def poisson_stream(rate=50.0, count=100, seed=0, widths=(512, 1024, 2048, 4096),
                   angles=(180, 720, 1500, 3000), max_slices=64):
    """Seeded request specs: (arrival s, n, nproj, nz, precision) with Poisson arrivals,
    uniform width/angle choices, nz ~ U{1..max_slices}, fp32 : mixed = 1 : 1."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    out = []
    for k in range(count):
        out.append((float(t[k]), int(rng.choice(widths)), int(rng.choice(angles)),
                    int(rng.integers(1, max_slices + 1)),
                    "float32" if k % 2 == 0 else "mixed"))
    return out
