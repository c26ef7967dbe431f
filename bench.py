#!/usr/bin/env python
"""Benchmark of the tomocupy_b200 reconstruction hot path.

Workload (production configuration): 2048 rows x 1500 angles over [0, pi) x
2048 columns of uint16 projections from a seeded synthetic ellipsoid phantom
(Poisson noise, 10 darks, 10 flats; the reference's APS datasets are not
available), dark/flat -> -log -> Shepp filter -> fourierrec, producing a
2048^3 float32 volume in device memory.  One step = the whole volume.

  value : GUPS (voxel*angle updates per second, n^2 * nz * nproj / t) with
          the frames already resident in HBM (12.6 GB input, larger than L2,
          so no flush is needed between steps).
  e2e   : the same metric through the public driver GPURec.recon_all with
          pinned HOST input and output (H2D of the frames and D2H of the
          volume inside the timed region).
  roofline : the dominant native kernel, timed with CUDA events recorded by
          the library around each launch on its stream.
  cpu_baseline : the NumPy port of the same steps on this host's cores,
          on a bounded sample (one slice pair), scaled to GUPS.

``--impl reference`` times the reference's own CUDA operators (built from the
reference sources into oracle/_ref) behind a torch restatement of its glue,
on the same workload and metric (a bounded slab per step).

N > 1 (torchrun): every rank reconstructs its own full volume (independent
datasets, no collective on the data path): weak scaling; NCCL is used only
for the barrier and the max-over-ranks of the step time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# algorithmic bytes per launch of each native stage (compulsory HBM traffic)
def stage_bytes(stage, n, nproj, ncz):
    ne = 4 * n
    pairs = ncz // 2
    table = {
        "prep_rows": ncz * nproj * n * (2 + 4),
        "filter_mulw": ncz * nproj * (ne // 2 + 1) * 16,
        "fr_pack": ncz * nproj * n * 4 + pairs * nproj * n * 8,
        "fr_gather": pairs * (nproj * n * 8 + (2 * n) ** 2 * 8),
        "fr_deapod": pairs * (n * n * 8 + 2 * n * n * 4),
        # own pruned 2D inverse FFT: rows pass (all 2n rows in, n kept columns
        # out), columns pass with deapodization (n columns in, n x n slices out)
        # fused filter: fp32 rows in, packed complex pairs (or their spectra) out
        "fft_filter": ncz * nproj * n * 4 + pairs * nproj * n * 8,
        "fr_ifft_rows": pairs * ((2 * n) ** 2 * 8 + 2 * n * n * 8),
        "fr_ifft_cols_deapod": pairs * (2 * n * n * 8 + 2 * n * n * 4),
        "fr_gather_tc": pairs * (nproj * n * 8 + (2 * n) ** 2 * 8),
        "linerec": ncz * (nproj * n * 4 + n * n * 8),
        # tensor-core filter: FLOPs (3 split products of 2 n^2 per row), not bytes
        "tc_filter": 3 * 2 * ncz * nproj * n * n,
    }
    return table.get(stage)


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per launch from
# the committed ncu captures, keyed by (stage, n, nproj, rows per chunk);
# see profiles/launches_fourierrec_pipeline_2048x1500.md and
# profiles/fr_gather_tc_grid_tc_2048x1500_32pairs.md
NCU_TRAFFIC = {("fr_gather", 2048, 1500, 64): 1216.8e6 + 4259.3e6,
               ("fft_filter", 2048, 1500, 64): 786.7e6 + 739.9e6,
               ("fr_ifft_cols_deapod", 2048, 1500, 64): 2149.4e6 + 1043.0e6,
               ("fr_ifft_rows", 2048, 1500, 64): 4295.0e6 + 2115.0e6,
               ("fr_gather_tc", 2048, 1500, 64): 1705.8e6 + 4260.5e6,
               # profiles/tc_filter_tcf_gemm_2048x1500_32slices.md
               ("tc_filter", 2048, 1500, 32): 411.44e6 + 359.14e6}


def setup_dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier_max(t_ms, ws):
    """Maximum of the ranks' device times (NCCL all-reduce when ws > 1)."""
    import torch
    from tomocupy_b200.multigpu import max_over_ranks
    return max_over_ranks(t_ms, torch.device("cuda", torch.cuda.current_device()))


def barrier(ws):
    import torch
    from tomocupy_b200.multigpu import barrier as mbarrier
    mbarrier(torch.device("cuda", torch.cuda.current_device()))


def make_data(a, device):
    from tomocupy_b200 import synthetic
    return synthetic.make_dataset(a.nproj, a.nz, a.n, seed=a.seed, device=device,
                                  block=32)


def cpu_model() -> str:
    """The host CPU's model name (the `lscpu` "Model name" field, read from
    /proc/cpuinfo so that no external tool is needed)."""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.lower().startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(a, data_cpu, dark, flat, theta):
    """NumPy port on the host cores: one slice pair through prep + filter + fourierrec."""
    from oracle import np_tomo
    z0 = a.nz // 2
    d = data_cpu[:, z0:z0 + 2]
    wf = np_tomo.calc_filter(4 * a.n, a.filter)  # filter spectrum: setup, not timed
    t0 = time.perf_counter()
    sino = np_tomo.minus_log(np_tomo.darkflat(d, dark[:, z0:z0 + 2], flat[:, z0:z0 + 2]))
    sino = np.ascontiguousarray(sino.transpose(1, 0, 2))
    filt = np_tomo.fbp_filter_center(sino, wf, a.n / 2, 0.0)
    np_tomo.fourierrec(filt, theta)
    secs = time.perf_counter() - t0
    gups = a.n * a.n * 2 * a.nproj / secs / 1e9
    return {"value": gups, "unit": "GUPS", "cores": np_tomo.WORKERS, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"1 slice pair of the {a.n}x{a.nproj} geometry (prep+filter+fourierrec, "
                      f"NumPy/scipy.fft float32, workers={np_tomo.WORKERS}), {secs:.1f} s",
            "seconds": secs}


def _time_path(a, ws, dtype, data, dark, flat, theta, dark0, flat0, out, dev, local):
    """Warm up, then time a.steps whole-volume reconstructions on the device."""
    import torch
    from tomocupy_b200 import _lib, global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    global_vars.reset(reconstruction_algorithm=a.algorithm, fbp_filter=a.filter,
                      nsino_per_chunk=a.ncz, dtype=dtype, **_ring_removal(a))
    rec = GPURec(ArrayReader(data, dark, flat, theta=theta), ArrayWriter(device=dev),
                 device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(a.warmup):
        rec.recon_device(data, dark0, flat0, out)
    barrier(ws)
    _lib.profile_enable(True)
    l0 = _lib.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(ws)
        ev0.record(stream)
        for _ in range(a.steps):
            rec.recon_device(data, dark0, flat0, out)
        ev1.record(stream)
        barrier(ws)
    launches = _lib.launch_count() - l0
    stages = _lib.profile_report()
    _lib.profile_enable(False)
    ms_step = barrier_max(ev0.elapsed_time(ev1), ws) / a.steps
    del rec
    return ms_step, stages, launches, clk.summary()


def _ring_removal(a):
    """Options of the Fourier-wavelet ring removal of the production pipeline."""
    if not a.ring_removal:
        return {}
    return dict(remove_stripe_method="fw", fw_sigma=1.0, fw_filter="sym16", fw_level=7)


def _stated(rec):
    """True when a stage's launches stated their algorithmic bytes."""
    return rec.get("bytes", 0) > 0


def _roofline(stages, a, peaks, peaks_kind, kernel=None):
    """Roofline of the dominant (or the named) native stage."""
    own = {k: v for k, v in stages.items()
           if _stated(v) or stage_bytes(k, a.n, a.nproj, a.ncz) is not None}
    dom = kernel if kernel in own else (max(own, key=lambda k: own[k]["ms"]) if own else None)
    if dom is None:
        return None
    per_launch_ms = own[dom]["ms"] / own[dom]["count"]
    if _stated(own[dom]):
        # the stage states its bytes (and FLOPs) per launch: the streamed
        # tensor-core gridding is bound by whichever of HBM and the tensor
        # pipe its launch needs longer on
        algo = own[dom]["bytes"] / own[dom]["count"]
        flops = own[dom].get("flops", 0) / own[dom]["count"]
        t_s = per_launch_ms / 1e3
        hbm = {"achieved": round(algo / t_s / 1e9, 1), "peak": peaks["hbm_gbs"],
               "unit": "GB/s", "frac": round(algo / t_s / 1e9 / peaks["hbm_gbs"], 4)}
        out = {"bound": "hbm", "kernel": dom, **hbm,
               "traffic": NCU_TRAFFIC.get((dom, a.n, a.nproj, a.ncz)),
               "algorithmic_bytes_per_launch": round(algo),
               "ms_per_launch": round(per_launch_ms, 4),
               "peak_source": f"{peaks_kind} (MEASURED_PEAKS.json hbm_gbs)"
               if peaks_kind == "measured" else "fallback 6.65 TB/s"}
        if flops > 0:
            tpeak = peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
            tfrac = flops / t_s / 1e12 / tpeak
            out["tensor"] = {"achieved": round(flops / t_s / 1e12, 1), "peak": tpeak,
                             "unit": "TFLOP/s", "frac": round(tfrac, 4),
                             "flops_per_launch": round(flops)}
            if tfrac > hbm["frac"]:  # the tensor pipe is the nearer bound
                out.update(bound="tensor", achieved=out["tensor"]["achieved"], peak=tpeak,
                           unit="TFLOP/s", frac=round(tfrac, 4))
        return out
    algo = stage_bytes(dom, a.n, a.nproj, a.ncz)
    if dom == "tc_filter":  # tensor-bound: algorithmic flops, fp16 dense = bf16 dense rate
        achieved = algo / (per_launch_ms / 1e3) / 1e12
        peak = peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
        return {"bound": "tensor", "kernel": dom, "achieved": round(achieved, 1),
                "peak": peak, "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                "traffic": NCU_TRAFFIC.get((dom, a.n, a.nproj, a.ncz)),
                "algorithmic_flops_per_launch": algo, "ms_per_launch": round(per_launch_ms, 4),
                "peak_source": (f"{peaks_kind} (MEASURED_PEAKS.json bf16_tflops_sustained, "
                                "kernel timed inside a long step)")
                if peaks_kind == "measured" else "fallback 1.4 PFLOP/s sustained"}
    achieved = algo / (per_launch_ms / 1e3) / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
            "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": round(achieved / peaks["hbm_gbs"], 4),
            "traffic": NCU_TRAFFIC.get((dom, a.n, a.nproj, a.ncz)),
            "algorithmic_bytes_per_launch": algo, "ms_per_launch": round(per_launch_ms, 4),
            "peak_source": f"{peaks_kind} (MEASURED_PEAKS.json hbm_gbs)"
            if peaks_kind == "measured" else "fallback 6.65 TB/s"}


def run_tc_filter(a, dev, peaks, peaks_kind, reps=10):
    """The tensor-core Toeplitz filter timed alone on one chunk of this workload.

    ncz slices x nproj rows x n columns (split fp16 operands, packed complex
    output), CUDA events around reps launches after 3 warm-ups; algorithmic
    flops 3 * 2 * n^2 per row against the burst bf16 peak (a kernel timed
    alone).  The pipelines use the fused FFT filter, which does O(n log n)
    work per row instead of the GEMM's O(n^2), so this leg reports the
    tensor-core kernel on its own.
    """
    import torch
    from tomocupy_b200.reconstruction.fbp_filter import calc_filter
    from tomocupy_b200.reconstruction.tcfilter import TCFilter, split16
    n, P, ncz = a.n, a.nproj, a.ncz
    g = torch.Generator(device=dev).manual_seed(a.seed)
    x = torch.rand((ncz, P, n), device=dev, generator=g)
    hi, lo = split16(x)
    f = TCFilter(n, P, ncz, 1, dev)
    f.set_kernels(calc_filter(4 * n, a.filter), 4 * n, n / 2)
    out = torch.empty((ncz // 2, P, n), dtype=torch.complex64, device=dev)
    s = torch.cuda.current_stream(dev)
    for _ in range(3):
        f.apply(hi, lo, out, pairs=True, stream=s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(s)
    for _ in range(reps):
        f.apply(hi, lo, out, pairs=True, stream=s)
    e1.record(s)
    torch.cuda.synchronize(dev)
    timed_out = f.timed_out()
    f.free()
    ms = e0.elapsed_time(e1) / reps
    flops = 3 * 2 * ncz * P * float(n) ** 2
    achieved = flops / (ms / 1e3) / 1e12
    peak = peaks["bf16_tflops"]
    return {"bound": "tensor", "kernel": "tc_filter", "timed": "alone",
            "workload": f"{ncz} slices x {P} rows x {n} columns, packed pair output",
            "achieved": round(achieved, 1), "peak": peak, "unit": "TFLOP/s",
            "frac": round(achieved / peak, 4),
            "traffic": NCU_TRAFFIC.get(("tc_filter", n, P, ncz)),
            "algorithmic_flops_per_launch": flops, "ms_per_launch": round(ms, 4),
            "timed_out": timed_out,
            "peak_source": f"{peaks_kind} (MEASURED_PEAKS.json bf16_tflops, burst: kernel "
                           "timed alone)" if peaks_kind == "measured" else "fallback 1.59 PFLOP/s"}


def run_try(a, dev):
    """Try-centre sweep: 1 slice x a.try_n cols x a.try_nproj angles x a.try_centers centres.

    Centres 2096 - 0.375 k (k < 256) around rotation axis 2048 for n = 4096;
    fourierrec, Parzen filter.  Each precision is autotuned (chunk size x
    gridding depth), captured as one CUDA graph and timed by graph replays.
    """
    import torch
    from tomocupy_b200 import synthetic
    from tomocupy_b200.processing.proc_functions import darkflat_stats
    from tomocupy_b200.trycenter import TryCenterSweep, autotune, per_center_errors
    n, P, S = a.try_n, a.try_nproj, a.try_centers
    data, dark, flat, theta, _ = synthetic.make_dataset(P, 1, n, seed=a.seed, device=dev)
    d0, f0, _ = darkflat_stats(dark, flat)
    center = n / 2
    shifts = (center + 48.0) - 0.375 * np.arange(S) - center  # centres 2096 - 0.375 k at n=4096
    shifts = -shifts  # the filter places the axis at center - sht
    res = {"workload": f"1 slice x {n} cols x {P} angles, {S} centres "
                       f"[{center + 48.0 - 0.375 * (S - 1):.3f}, {center + 48.0:.3f}] step 0.375",
           "unit": "GUPS (n^2 * nproj * centres / t)"}
    outs = {}
    for prec in ("float32", "mixed"):
        tune = autotune(n, P, theta, center, shifts, data, d0, f0, fbp_filter="parzen",
                        precision=prec, candidates=[(32, 16), (64, 16), (128, 16)], reps=1)
        sw = TryCenterSweep(n, P, theta, center, shifts, "parzen", prec, tune["ncz"],
                            tune["pairs_per_block"], dev)
        sw.load(data, d0, f0)
        sw.capture()
        sw.time_ms(1)
        ms = sw.time_ms(3)
        outs[prec] = sw.run().clone()
        res[prec] = {"ms_per_sweep": round(ms, 3),
                     "value": round(float(n) ** 2 * P * S / (ms / 1e3) / 1e9, 2),
                     "graph_launches_per_sweep": 1, "ncz": tune["ncz"],
                     "pairs_per_block": tune["pairs_per_block"], "autotune": tune["table"]}
        sw.free()
        del sw
        torch.cuda.empty_cache()
    rel, mx = per_center_errors(outs["mixed"].cpu(), outs["float32"].cpu())
    res["mixed_vs_fp32_per_center"] = {"rel_l2_max": float(rel.max()),
                                       "rel_l2_median": float(np.median(rel)),
                                       "max_abs_max": float(mx.max())}
    res["mixed_speedup_vs_fp32"] = round(res["float32"]["ms_per_sweep"] /
                                         res["mixed"]["ms_per_sweep"], 3)
    res["fp64_oracle"] = ("per-centre rel-L2 vs FP64 in "
                          "tests/test_gpu_trycenter.py::test_mixed_sweep_vs_fp64_oracle_per_center")
    del outs
    torch.cuda.empty_cache()
    return res


def run_serving(a, dev):
    """Serving leg: a seeded Poisson stream of uneven reconstructions.

    Arrivals at a.serve_rate req/s; width from {512, 1024, 2048, 4096},
    angles from {180, 720, 1500, 3000}, slices U{1..64}, uint16 frames,
    fp32 : mixed = 1 : 1.  Frames come from pinned host stacks (one per
    width x angles, 64 slices; a request takes a slab), results go to pinned
    host buffers.  Geometries are made resident before the stream.
    """
    import torch
    from tomocupy_b200 import synthetic
    from tomocupy_b200.serving import Request, Server, latency_summary, poisson_stream
    specs = poisson_stream(rate=a.serve_rate, count=a.serve_requests, seed=a.seed)
    pool = {}
    for _, n, P, _, _ in specs:
        if (n, P) not in pool:
            d, dk, fl, th, _ = synthetic.make_dataset(P, 64, n, seed=a.seed, device=dev)
            pool[(n, P)] = (d.cpu().pin_memory(), dk.cpu().pin_memory(), fl.cpu().pin_memory(),
                            th)
            del d, dk, fl
    # every request writes its own pinned host volume (sized for fp32, viewed as
    # fp16 for mixed requests), so concurrent requests never copy into the same
    # host memory; with too little host memory, a ring of buffers per width
    # that is longer than the server's admission limit
    need = sum(nz * n * n * 4 for _, n, _, nz, _ in specs)
    own = need * 1.5 < _mem_available()
    ring = {}
    outs = []
    for k, (_, n, _, nz, _) in enumerate(specs):
        if own:
            outs.append(torch.empty(nz * n * n * 4, dtype=torch.uint8, pin_memory=True))
        else:
            r = ring.setdefault(n, [])
            if len(r) < 32:
                r.append(torch.empty(64 * n * n * 4, dtype=torch.uint8, pin_memory=True))
            outs.append(r[sum(1 for _, m, _, _, _ in specs[:k] if m == n) % 32])

    def make(precision=None):
        # mixed-precision requests return fp16 volumes, fp32 requests fp32
        reqs = []
        for k, (t, n, P, nz, prec) in enumerate(specs):
            d, dk, fl, th = pool[(n, P)]
            prec = precision or prec
            odt = "float16" if prec == "mixed" else "float32"
            dt = torch.float16 if odt == "float16" else torch.float32
            out = outs[k].view(dt)[:nz * n * n].view(nz, n, n)
            reqs.append(Request(k, d[:, :nz], dk[:, :nz], fl[:, :nz], th, n / 2, prec, "parzen",
                                arrival=t, out=out, out_dtype=odt))
        return reqs

    res = {"workload": f"{len(specs)} requests, Poisson {a.serve_rate}/s (seed {a.seed}), "
                       "n in {512,1024,2048,4096}, nproj in {180,720,1500,3000}, nz U{1..64}, "
                       "fp32:mixed 1:1 (mixed requests return fp16 volumes), uint16 pinned host "
                       "frames -> pinned host volumes",
           "hbm_budget_gb": a.serve_budget_gb,
           "output_buffers": "one per request" if own else "ring of 32 per width"}
    srv = Server(dev, hbm_budget=a.serve_budget_gb * 1e9, ncz=a.serve_ncz)
    srv.warm(make())
    srv.warm(make("float32"))
    # single-request latency: each request alone on the warm server
    alone = make()
    for r in alone:
        r.arrival = 0.0
        srv.serve([r], realtime=False)
    single = np.array([r.latency for r in alone]) * 1e3
    res["single_request"] = {"p50_ms": float(np.percentile(single, 50)),
                             "p99_ms": float(np.percentile(single, 99))}
    mix = make()
    srv.serve(mix, realtime=True)
    res["continuous_batching"] = latency_summary(mix)
    res["continuous_batching"]["peak_admitted"] = srv.peak_active
    res["continuous_batching"]["peak_resident_gb"] = round(srv.peak_bytes / 1e9, 2)
    # same-geometry requests packed into shared chunk launches
    res["continuous_batching"]["chunk_launches"] = srv.chunks
    res["continuous_batching"]["chunks_one_request_each"] = int(sum(
        -(-m.frames.shape[1] // a.serve_ncz) for m in mix))
    ratio = np.array([m.latency / s.latency for m, s in zip(mix, alone)])
    res["latency_in_mix_over_alone"] = {"p50": float(np.percentile(ratio, 50)),
                                        "p99": float(np.percentile(ratio, 99))}
    res["p99_over_single_p99"] = round(res["continuous_batching"]["p99_ms"] /
                                       res["single_request"]["p99_ms"], 3)
    base = Server(dev, hbm_budget=a.serve_budget_gb * 1e9, ncz=a.serve_ncz, max_active=1)
    base.geoms = srv.geoms  # same resident geometries
    base.geom_bytes = srv.geom_bytes
    seq = make("float32")
    base.serve(seq, realtime=True)
    res["one_at_a_time_fp32"] = latency_summary(seq)
    res["GUPS_vs_one_at_a_time_fp32"] = round(res["continuous_batching"]["GUPS"] /
                                              res["one_at_a_time_fp32"]["GUPS"], 3)
    del srv, base, pool, outs
    torch.cuda.empty_cache()
    return res


def _lamino_setup(a, dtype):
    from tomocupy_b200 import global_vars
    from tomocupy_b200.global_vars import params
    ntheta, n, rh, tilt = a.lam_nproj, a.lam_n, a.lam_rh, 30.0
    theta = (np.arange(ntheta) * 2 * np.pi / ntheta).astype(np.float32)
    global_vars.reset(lamino_angle=tilt, reconstruction_algorithm="fourierrec",
                      nsino_per_chunk=32, nproj_per_chunk=60, fbp_filter="shepp", dtype=dtype)
    params.n, params.nz, params.nproj, params.ncproj, params.ncz = n, n, ntheta, 60, 32
    params.rh, params.center, params.theta, params.lamino_angle = rh, n / 2, theta, tilt
    return theta


def _lamino_data(a, dev):
    """Seeded smooth projections [nproj, n, n] (content does not change the timing)."""
    import torch
    from tomocupy_b200.synthetic import smooth_field
    gen = torch.Generator(device=dev)
    gen.manual_seed(a.seed)
    base = smooth_field(a.lam_n, a.lam_n, 24.0, gen, dev).abs()
    ang = torch.arange(a.lam_nproj, device=dev, dtype=torch.float32)
    return (base[None] * (1.0 + 0.1 * torch.cos(ang * 2 * np.pi / a.lam_nproj))[:, None, None]
            ).contiguous()


def run_lamino(a, dev):
    """Laminography leg: fp32 chain and fp16 stage storage, device-resident."""
    import torch
    from tomocupy_b200.reconstruction.backproj_lamfourier_parallel import \
        BackprojLamFourierParallel
    data = _lamino_data(a, dev)
    vox = float(a.lam_rh) * a.lam_n * a.lam_n * a.lam_nproj
    res = {"workload": f"{a.lam_nproj} angles over [0, 2pi) x {a.lam_n}^2 fp32 projections, "
                       f"tilt 30 deg, rh {a.lam_rh} -> {a.lam_rh}x{a.lam_n}^2 volume "
                       "(seeded smooth projections)", "unit": "GUPS (rh*n^2*nproj/t)"}
    outs = {}
    for dtype in ("float32", "mixed"):
        _lamino_setup(a, dtype)
        bp = BackprojLamFourierParallel(device=dev)
        bp.rec_lam(data)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(2):
            out = bp.rec_lam(data)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 2
        from tomocupy_b200 import _lib
        _lib.profile_enable(True)
        bp.rec_lam(data)
        stages = _lib.profile_report()
        _lib.profile_enable(False)
        key = "fp32" if dtype == "float32" else "fp16_storage"
        res[key] = {"ms": round(ms, 2), "value": round(vox / (ms / 1e3) / 1e9, 2),
                    "stages_ms": {k: round(v["ms"], 2) for k, v in stages.items()}}
        outs[key] = out
        del bp
    d = (outs["fp16_storage"].double() - outs["fp32"].double()).norm()
    res["fp16_storage_rel_l2_vs_fp32"] = float(d / outs["fp32"].double().norm())
    del outs, data
    torch.cuda.empty_cache()
    return res


def run_methods(a, data, dark, flat, theta, dev):
    """The rest of the production configuration, fp32 drop-in path, frames resident:
    fourierrec with Fourier-wavelet ring removal (level 7, sigma 1, sym16) and with
    Titarenko ring removal (beta 0.022, full mask) and with outlier removal
    (dezinger width 3, threshold 5000) on the whole volume, and lprec / linerec on
    a bounded slab of rows."""
    import torch
    from tomocupy_b200 import _lib, global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.processing.proc_functions import darkflat_stats
    from tomocupy_b200.rec import GPURec
    res = {}
    legs = [("fourierrec+fw", "fourierrec", a.nz, dict(remove_stripe_method="fw", fw_sigma=1.0,
                                                         fw_filter="sym16", fw_level=7)),
            ("fourierrec+ti", "fourierrec", a.nz, dict(remove_stripe_method="ti", ti_beta=0.022,
                                                         ti_mask=1)),
            ("fourierrec+dezinger", "fourierrec", a.nz, dict(dezinger=3,
                                                              dezinger_threshold=5000)),
            ("fourierrec+vo-all", "fourierrec", min(a.nz, a.slab_rows),
             dict(remove_stripe_method="vo-all")),
            ("lprec", "lprec", min(a.nz, a.slab_rows), {}),
            ("linerec", "linerec", min(a.nz, a.slab_rows), {})]
    for name, alg, rows, extra in legs:
        d, dk, fl = data[:, :rows], dark[:, :rows], flat[:, :rows]
        # lprec and linerec keep 64-row chunks (their kernels gain nothing from more)
        global_vars.reset(reconstruction_algorithm=alg, fbp_filter=a.filter,
                          nsino_per_chunk=a.ncz if alg == "fourierrec" else min(a.ncz, 64),
                          **extra)
        rec = GPURec(ArrayReader(d, dk, fl, theta=theta), ArrayWriter(device=dev), device=dev)
        d0, f0, _ = darkflat_stats(dk, fl)
        out = torch.empty((params.nz, params.n, params.n), dtype=torch.float32, device=dev)
        rec.recon_device(d, d0, f0, out)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rec.recon_device(d, d0, f0, out)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        _lib.profile_enable(True)
        rec.recon_device(d, d0, f0, out)
        stages = _lib.profile_report()
        _lib.profile_enable(False)
        res[name] = {"rows": rows, "ms": round(ms, 2), "unit": "GUPS",
                     "value": round(float(a.n) ** 2 * rows * a.nproj / (ms / 1e3) / 1e9, 2),
                     "stages_ms": {k: round(v["ms"], 2) for k, v in stages.items()}}
        del rec, out
        torch.cuda.empty_cache()
    return res


def run_phase(a, dev, peaks, peaks_kind):
    """Paganin phase retrieval of 2048 x 2048 projections (a.phase_proj of them,
    frames resident) with production optics: 0.65 um pixels, 50 mm, 20 keV ->
    4096 x 4096 padded transforms.  Algorithmic bytes: 8 per detector pixel
    (float32 read + write); the padded chain's own traffic is in the stages."""
    import torch
    from oracle import np_tomo
    from tomocupy_b200 import _lib
    from tomocupy_b200.processing.retrieve_phase import PhaseFilter
    n, P = a.n, a.phase_proj
    ps, dist, en, alpha = 0.65e-4, 5.0, 20.0, 1e-3
    g = torch.Generator(device=dev).manual_seed(a.seed)
    x = 0.5 + 0.4 * torch.rand((P, n, n), device=dev, generator=g)
    op = PhaseFilter(n, n, "paganin", ps, dist, en, alpha)
    y = x.clone()
    for _ in range(2):
        op.apply(y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    e0.record()
    for _ in range(reps):
        op.apply(y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    _lib.profile_enable(True)
    op.apply(y)
    stages = _lib.profile_report()
    _lib.profile_enable(False)
    # parity of the first projection against the NumPy restatement
    want = np_tomo.retrieve_phase(x[:1].cpu().numpy(), "paganin", ps, dist, en, alpha)
    y1 = op.apply(x[:1].clone()).cpu().numpy()
    rel = float(np.linalg.norm(y1 - want) / np.linalg.norm(want))
    t0 = time.perf_counter()
    np_tomo.retrieve_phase(x[:1].cpu().numpy(), "paganin", ps, dist, en, alpha)
    cpu_s = time.perf_counter() - t0
    alg = 8.0 * P * n * n
    # the three-pass chain's traffic (pairs of projections packed as one
    # complex image): rows pass reads the two images and writes the padded
    # row spectra (8 B per padded pixel), the columns pass reads them and
    # writes the dy kept rows (8 B per kept-row pixel), the last rows pass
    # reads those and writes the two images
    Ny, Nz = n + 2 * op.py, n + 2 * op.pz
    chain = (P / 2.0) * (2 * 4.0 * n * n + 2 * 8.0 * Ny * Nz + 2 * 8.0 * n * Nz +
                         2 * 4.0 * n * n)
    res = {"workload": f"{P} projections {n}x{n} float32, paganin (0.65 um, 50 mm, 20 keV, "
                       f"alpha 1e-3), padded {n + 2 * op.py}x{n + 2 * op.pz}",
           "ms": round(ms, 2), "projections_per_s": round(P / (ms / 1e3), 1),
           "unit": "projections/s", "batch": op.batch,
           "achieved_gbs_algorithmic": round(alg / (ms / 1e3) / 1e9, 1),
           "padded_chain_bytes": chain,
           "achieved_gbs_padded_chain": round(chain / (ms / 1e3) / 1e9, 1),
           "peak_gbs": peaks.get("hbm_gbs"), "peak_source": peaks_kind,
           "stages_ms": {k: round(v["ms"], 2) for k, v in stages.items()},
           "rel_l2_vs_numpy_oracle_first_projection": rel,
           "cpu_baseline": {"value": round(1.0 / cpu_s, 3), "unit": "projections/s",
                            "kind": "port", "cores": 1,
                            "sample": f"1 projection {n}x{n} (NumPy complex64 fft2/ifft2 as "
                                      f"the reference), {cpu_s:.1f} s"}}
    # projection rotation (rotate_proj, order 1, 1 degree) of the same stack:
    # 8 algorithmic bytes per pixel (float32 read + write), 1 GiB in and out
    from tomocupy_b200.processing.proc_functions import rotate_proj
    for _ in range(3):
        rotate_proj(x, 1.0, 1, out=y)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        rotate_proj(x, 1.0, 1, out=y)
    e1.record()
    torch.cuda.synchronize()
    rms = e0.elapsed_time(e1) / reps
    want = np_tomo.rotate_proj(x[:1].cpu().numpy(), 1.0, 1)
    exact = bool(np.array_equal(y[:1].cpu().numpy(), want))
    t0 = time.perf_counter()
    np_tomo.rotate_proj(x[:1].cpu().numpy(), 1.0, 1)
    rcpu = time.perf_counter() - t0
    ragb = alg / (rms / 1e3) / 1e9
    res["rotate"] = {
        "workload": f"{P} projections {n}x{n} float32, 1 degree, spline order 1, 'nearest'",
        "ms": round(rms, 3), "projections_per_s": round(P / (rms / 1e3), 1),
        "roofline": {"bound": "hbm", "achieved": round(ragb, 1), "peak": peaks.get("hbm_gbs"),
                     "unit": "GB/s", "frac": round(ragb / peaks["hbm_gbs"], 3)
                     if peaks.get("hbm_gbs") else None, "peak_source": peaks_kind},
        "bit_exact_vs_numpy_oracle_first_projection": exact,
        "cpu_baseline": {"value": round(1.0 / rcpu, 3), "unit": "projections/s",
                         "kind": "port", "cores": 1,
                         "sample": f"1 projection {n}x{n} (NumPy float64), {rcpu:.2f} s"}}
    op.free()
    del x, y
    torch.cuda.empty_cache()
    return res


def run_ours(a, ws, rank, local):
    import torch
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.processing.proc_functions import darkflat_stats

    dev = torch.device("cuda", local)
    t_gen = time.perf_counter()
    data, dark, flat, theta, _ = make_data(a, dev)
    torch.cuda.synchronize()
    log(f"[rank {rank}] generated {tuple(data.shape)} in {time.perf_counter() - t_gen:.1f} s")
    dark0, flat0, _ = darkflat_stats(dark, flat)
    out = torch.empty((a.nz, a.n, a.n), dtype=torch.float32, device=dev)
    peaks, peaks_kind = load_peaks()
    vox = float(a.n) ** 2 * a.nz * a.nproj

    # primary path (the drop-in fp32 by default) and the other precision beside it
    primary = a.precision
    other = "mixed" if primary == "float32" else "float32"
    ms_step, stages, launches, clocks = _time_path(a, ws, primary, data, dark, flat, theta,
                                                   dark0, flat0, out, dev, local)
    value = ws * vox / (ms_step / 1e3) / 1e9
    slices_s = ws * a.nz / (ms_step / 1e3)
    roofline = _roofline(stages, a, peaks, peaks_kind)
    side = None
    if not a.no_mixed:
        out2 = torch.empty_like(out)
        ms2, st2, l2, clk2 = _time_path(a, ws, other, data, dark, flat, theta, dark0, flat0,
                                        out2, dev, local)
        # whole-volume agreement of the two precisions (both outputs resident)
        diff = 0.0
        ref2 = 0.0
        for z0 in range(0, a.nz, 64):
            diff += float(torch.sum((out2[z0:z0 + 64] - out[z0:z0 + 64]).double() ** 2))
            ref2 += float(torch.sum(out[z0:z0 + 64].double() ** 2))
        del out2
        v2 = ws * vox / (ms2 / 1e3) / 1e9
        mixed_ms, fp32_ms = (ms2, ms_step) if other == "mixed" else (ms_step, ms2)
        side = {"precision": other, "value": round(v2, 2), "unit": "GUPS",
                "ms_per_step": round(ms2, 3), "slices_per_s": round(ws * a.nz / (ms2 / 1e3), 1),
                "mixed_speedup_vs_fp32": round(fp32_ms / mixed_ms, 3),
                "rel_l2_vs_" + primary: math.sqrt(diff / max(ref2, 1e-300)),
                "rel_l2_vs_fp64": "see tests/test_gpu_pipeline.py::"
                                  "test_c1_mixed_fourierrec_vs_fp64_oracle (budget 1e-3)",
                "gpu_launches": l2, "clocks": clk2,
                "roofline_tc_filter": run_tc_filter(a, dev, peaks, peaks_kind),
                "stages_ms": {k: round(v["ms"] / a.steps, 3) for k, v in st2.items()}}

    methods = None
    if not a.no_methods and ws == 1:
        methods = run_methods(a, data, dark, flat, theta, dev)

    # ---------------- e2e through the public driver with host buffers
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(a, data, dark, flat, theta, dev, ws, rank)
        if side is not None and ws == 1:
            # the mixed path end to end, with fp16 output slices (half the D2H bytes)
            side["e2e_fp16_out"] = run_e2e(a, data, dark, flat, theta, dev, ws, rank,
                                           precision="mixed", out_dtype="float16")

    # the e2e legs' pinned host stacks stay in torch's host cache otherwise
    if hasattr(torch._C, "_host_emptyCache"):
        torch._C._host_emptyCache()

    base = None
    if rank == 0 and ws == 1 and not a.no_cpu:
        dcpu, dkc, flc = data.cpu().numpy(), dark.cpu().numpy(), flat.cpu().numpy()
        base = cpu_baseline(a, dcpu, dkc, flc, theta)
        del dcpu, dkc, flc

    # the remaining legs need the device memory of the volume workload
    del out, data, dark, flat, dark0, flat0
    torch.cuda.empty_cache()
    trycenter = None
    if not a.no_try and ws == 1:
        trycenter = run_try(a, dev)
    serving = None
    if not a.no_serve and ws == 1:
        serving = run_serving(a, dev)
        if hasattr(torch._C, "_host_emptyCache"):
            torch._C._host_emptyCache()
    lamino = None
    if not a.no_lamino and ws == 1:
        lamino = run_lamino(a, dev)
    phase = None
    if not a.no_phase and ws == 1:
        phase = run_phase(a, dev, peaks, peaks_kind)

    if rank == 0:
        tag = "fp32" if primary == "float32" else "mixed-precision"
        line = {
            "metric": f"GUPS @{a.n}^2x{a.nproj} ({a.algorithm} {tag} pipeline, 1 GPU rate)",
            "value": round(value, 2), "unit": "GUPS", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if primary == "float32" else "f16x2 operands / f32 accumulate",
            "data": "synthetic",
            "config": {"workload": f"{a.nz} rows x {a.nproj} angles x {a.n} cols uint16 -> "
                                   f"{a.nz}x{a.n}^2 f32 volume; dark/flat, -log, {a.filter} "
                                   f"filter, {a.algorithm}; ring removal "
                                   f"{'fw level 7 sigma 1 sym16' if a.ring_removal else 'off'}",
                       "n": a.n, "nproj": a.nproj, "nz": a.nz, "ncz": a.ncz,
                       "e2e_ncz": a.e2e_ncz,
                       "precision": primary,
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "inputs (12.6 GB frames) larger than L2; no flush"},
            "slices_per_s": round(slices_s, 1),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": base,
            "clocks": clocks, "gpu_launches": launches,
            "stages_ms": {k: round(v["ms"] / a.steps, 3) for k, v in stages.items()},
            other if other == "mixed" else "fp32": _compact(side),
            "methods": methods,
            "try_center": _compact(trycenter),
            "serving": _compact(serving),
            "lamino": _compact(lamino),
            "phase_retrieval": _compact(phase),
        }
        line["summary"] = _summary(line, side, methods, trycenter, serving, lamino, phase)
        # the full records of the side legs (autotune tables, per-stage times) go to
        # stderr; the JSON line on stdout stays short and ends with the summary
        log("detail: " + json.dumps({"mixed": side, "try_center": trycenter, "serving": serving,
                                     "lamino": lamino, "phase_retrieval": phase}))
        print(json.dumps(line), flush=True)


_VERBOSE = ("autotune", "stages_ms", "workload", "peak_source", "fp64_oracle",
            "rel_l2_vs_fp64", "api", "sample")


def _compact(d):
    """A leg's record without its long descriptive fields (kept on stderr)."""
    if not isinstance(d, dict):
        return d
    return {k: _compact(v) for k, v in d.items() if k not in _VERBOSE}


def _summary(line, side, methods, trycenter, serving, lamino, phase):
    """The figures of every leg in one short object at the end of the line."""
    g = lambda d, *ks: _dig(d, ks)  # noqa: E731
    return {
        "fp32_gups": line["value"], "fp32_ms": line["ms_per_step"],
        "e2e_gups": g(line, "e2e", "value"),
        "roofline_kernel": g(line, "roofline", "kernel"),
        "roofline_frac": g(line, "roofline", "frac"),
        "mixed_gups": g(side, "value"), "mixed_ms": g(side, "ms_per_step"),
        "mixed_speedup_vs_fp32": g(side, "mixed_speedup_vs_fp32"),
        "mixed_rel_l2_vs_fp32": g(side, "rel_l2_vs_float32"),
        "mixed_e2e_fp16_out_gups": g(side, "e2e_fp16_out", "value"),
        "fw_gups": g(methods, "fourierrec+fw", "value"),
        "fw_ms": g(methods, "fourierrec+fw", "ms"),
        "ti_gups": g(methods, "fourierrec+ti", "value"),
        "dezinger_gups": g(methods, "fourierrec+dezinger", "value"),
        "vo_all_gups": g(methods, "fourierrec+vo-all", "value"),
        "lprec_gups": g(methods, "lprec", "value"),
        "linerec_gups": g(methods, "linerec", "value"),
        "try_fp32_ms": g(trycenter, "float32", "ms_per_sweep"),
        "try_mixed_ms": g(trycenter, "mixed", "ms_per_sweep"),
        "try_mixed_speedup": g(trycenter, "mixed_speedup_vs_fp32"),
        "serve_p50_ms": g(serving, "continuous_batching", "p50_ms"),
        "serve_p99_ms": g(serving, "continuous_batching", "p99_ms"),
        "serve_single_p99_ms": g(serving, "single_request", "p99_ms"),
        "serve_p99_over_single_p99": g(serving, "p99_over_single_p99"),
        "lamino_fp32_ms": g(lamino, "fp32", "ms"),
        "lamino_fp16_storage_ms": g(lamino, "fp16_storage", "ms"),
        "phase_projections_per_s": g(phase, "projections_per_s"),
        "fw_taps": "derived by spectral factorisation (PyWavelets absent): parity with "
                   "PyWavelets' sym16 table unpinned",
    }


def _dig(d, keys):
    for k in keys:
        if not isinstance(d, dict) or k not in d:
            return None
        d = d[k]
    return round(d, 4) if isinstance(d, float) else d


def _mem_available() -> int:
    """Host memory available to this process (bytes, /proc/meminfo)."""
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return 0


def run_e2e(a, data, dark, flat, theta, dev, ws, rank, precision=None, out_dtype="float32"):
    import torch
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    avail = _mem_available()
    osz = 2 if out_dtype == "float16" else 4
    full_bytes = data.numel() * 2 + a.nz * a.n * a.n * osz
    nz_e2e = a.nz if (avail > 3 * full_bytes * ws) else min(a.nz, a.e2e_slab)
    ncz = a.e2e_ncz  # the conveyor overlaps copies chunk by chunk: smaller chunks fill sooner
    nz_e2e -= nz_e2e % ncz
    d_host = data[:, :nz_e2e].cpu().pin_memory()
    dk_host = dark[:, :nz_e2e].cpu().pin_memory()
    fl_host = flat[:, :nz_e2e].cpu().pin_memory()
    global_vars.reset(reconstruction_algorithm=a.algorithm, fbp_filter=a.filter,
                      nsino_per_chunk=ncz, dtype=precision or a.precision, out_dtype=out_dtype,
                      **_ring_removal(a))
    reader = ArrayReader(d_host, dk_host, fl_host, theta=theta)
    writer = ArrayWriter(device="cpu", pin=True,
                         dtype=torch.float16 if out_dtype == "float16" else torch.float32)
    rec = GPURec(reader, writer, device=dev)
    for _ in range(max(1, min(a.warmup, 2))):
        rec.recon_all()
    stream = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    t0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(a.steps):
        rec.recon_all()  # ends with a device synchronize
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / a.steps
    ms = barrier_max(ev0.elapsed_time(ev1) / a.steps, ws)
    vox = float(a.n) ** 2 * nz_e2e * a.nproj
    h2d = d_host.numel() * 2 + dk_host.numel() * 2 + fl_host.numel() * 2
    d2h = nz_e2e * a.n * a.n * osz
    return {"value": round(ws * vox / (ms / 1e3) / 1e9, 2), "unit": "GUPS",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "rows": nz_e2e, "rows_per_chunk": ncz, "ms_per_step": round(ms, 2),
            "wall_ms_per_step": round(wall * 1e3, 2),
            # the bound of this leg: the host link, one direction each way
            "d2h_gbs": round(d2h / (ms / 1e3) / 1e9, 1),
            "h2d_gbs": round(h2d / (ms / 1e3) / 1e9, 1),
            "api": "GPURec.recon_all (pinned host frames -> pinned host volume)",
            "precision": precision or a.precision, "out_dtype": out_dtype}


def run_reference(a, ws, rank, local):
    """The reference's CUDA operators (oracle/_ref) behind its restated glue."""
    import torch
    if rank != 0:
        return
    from oracle import np_tomo, refglue
    if not refglue.available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    dev = torch.device("cuda", local)
    rows = min(a.nz, a.ref_rows)
    aa = argparse.Namespace(**vars(a))
    aa.nz = rows
    data, dark, flat, theta, _ = make_data(aa, dev)
    n, P, ncz = a.n, a.nproj, 8  # the reference default nsino_per_chunk
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, a.filter), device=dev)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=dev)
    th = torch.as_tensor(theta, device=dev)
    filt = refglue.RefFilter(ne, P, ncz)
    center = n / 2
    if a.algorithm == "fourierrec":
        op = refglue.RefFourierRec(n, P, ncz, th)
    elif a.algorithm == "lprec":
        from tomocupy_b200.reconstruction import lprec_grids as L
        ntheta, nrho = L.lp_sizes(n, P)
        op = refglue.RefLpRec(n, P, ncz, vars(L.create_adj(L.create_gl(n, P, ntheta, nrho))))
        center += 0.5
    else:
        op = refglue.RefLineRec(th, P, P, ncz, ncz, n)
    out = torch.zeros((rows, n, n), dtype=torch.float32, device=dev)

    def step():
        for z0 in range(0, rows, ncz):
            d = refglue.ref_darkflat_minus_log(data[:, z0:z0 + ncz], dark[:, z0:z0 + ncz],
                                               flat[:, z0:z0 + ncz])
            d = d.permute(1, 0, 2).contiguous()
            d = refglue.ref_fbp_filter_center(filt, d, wf, t, center, 0.0, n, ne)
            op.backprojection(out[z0:z0 + ncz], d)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(a.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / a.steps
    value = float(n) ** 2 * rows * P / (ms / 1e3) / 1e9
    lam = None
    if not a.no_lamino:
        _lamino_setup(a, "float32")
        ld = _lamino_data(a, dev)
        th = torch.as_tensor((np.arange(a.lam_nproj) * 2 * np.pi / a.lam_nproj).astype(np.float32),
                             device=dev)
        wl = torch.as_tensor(np_tomo.calc_filter(4 * a.lam_n, "shepp"), device=dev)
        refglue.ref_rec_lam(ld, th, a.lam_n / 2, 30.0, a.lam_rh, wl, nthetac=60, dethc=32, n1c=32)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        refglue.ref_rec_lam(ld, th, a.lam_n / 2, 30.0, a.lam_rh, wl, nthetac=60, dethc=32, n1c=32)
        e1.record()
        torch.cuda.synchronize()
        lms = e0.elapsed_time(e1)
        lam = {"ms": round(lms, 2), "unit": "GUPS (rh*n^2*nproj/t)",
               "value": round(float(a.lam_rh) * a.lam_n ** 2 * a.lam_nproj / (lms / 1e3) / 1e9, 2),
               "workload": "laminography, same as our lamino leg (reference CUDA operators)"}
        del ld
    others = {} if a.no_methods else _reference_methods(a, data, dark, flat, theta, dev)
    line = {"impl": "reference",
            "metric": f"GUPS @{a.n}^2x{a.nproj} ({a.algorithm} fp32 pipeline, 1 GPU rate)",
            "value": round(value, 2), "unit": "GUPS", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{rows}-row slab of the {a.nz} rows x {a.nproj} angles x "
                                   f"{a.n} cols workload; dark/flat, -log, {a.filter}, "
                                   f"{a.algorithm}", "n": n, "nproj": P, "rows_per_step": rows,
                       "ncz": ncz},
            "cpu_baseline": {"value": round(value, 2), "unit": "GUPS", "cores": 1,
                             "kind": "reference",
                             "sample": f"reference CUDA build (sources compiled for sm_100a) "
                                       f"on the B200, {rows} rows per step, driven by 1 host "
                                       f"thread; the reference has no CPU implementation"},
            "e2e": {"value": round(value, 2), "unit": "GUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "lamino": lam,
            "summary": {"fourierrec_fp32_gups": round(value, 2), **others,
                        "lamino_ms": lam["ms"] if lam else None}}
    print(json.dumps(line), flush=True)


def _reference_methods(a, data, dark, flat, theta, dev):
    """The reference's other operators on slabs of the same workload, each
    timed once after one warm-up run: its -DHALF fourierrec build with its
    fp16 filter (the reference's own fast path, the anchor of our mixed
    precision), lprec and linerec.  Reported in GUPS (n^2 rows nproj / t)."""
    import torch
    from oracle import np_tomo, refglue
    n, P = a.n, a.nproj
    ne = 4 * n
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=dev)
    th = torch.as_tensor(theta, device=dev)
    res = {}
    legs = [("fourierrec_fp16", 64, 8), ("lprec", 64, 8), ("linerec", 16, 8)]
    for name, rows, ncz in legs:
        rows = min(rows, data.shape[1])
        center = n / 2
        if name == "fourierrec_fp16":
            filt = refglue.RefFilter(ne, P, ncz, "float16")
            op = refglue.RefFourierRec(n, P, ncz, th, "float16")
            wf = torch.as_tensor(np_tomo.calc_filter(ne, a.filter), device=dev)
        elif name == "lprec":
            from tomocupy_b200.reconstruction import lprec_grids as L
            ntheta, nrho = L.lp_sizes(n, P)
            filt = refglue.RefFilter(ne, P, ncz)
            op = refglue.RefLpRec(n, P, ncz, vars(L.create_adj(L.create_gl(n, P, ntheta, nrho))))
            wf = torch.as_tensor(np_tomo.calc_filter(ne, a.filter), device=dev)
            center += 0.5
        else:
            filt = refglue.RefFilter(ne, P, ncz)
            op = refglue.RefLineRec(th, P, P, ncz, ncz, n)
            wf = torch.as_tensor(np_tomo.calc_filter(ne, a.filter), device=dev)
        half = name == "fourierrec_fp16"
        out = torch.zeros((ncz, n, n), dtype=torch.float16 if half else torch.float32,
                          device=dev)

        def step():
            for z0 in range(0, rows, ncz):
                d = refglue.ref_darkflat_minus_log(data[:, z0:z0 + ncz], dark[:, z0:z0 + ncz],
                                                   flat[:, z0:z0 + ncz])
                d = d.permute(1, 0, 2).contiguous()
                if half:
                    d = refglue.ref_fbp_filter_center(filt, d.half(), wf, t, center, 0.0, n,
                                                      ne)
                else:
                    d = refglue.ref_fbp_filter_center(filt, d, wf, t, center, 0.0, n, ne)
                op.backprojection(out, d)
        step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[name + "_gups"] = round(float(n) ** 2 * rows * P / (ms / 1e3) / 1e9, 2)
        res[name + "_rows"] = rows
        del op, filt, out
        torch.cuda.empty_cache()
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--nproj", type=int, default=1500)
    ap.add_argument("--nz", type=int, default=2048)
    ap.add_argument("--ncz", type=int, default=128)
    ap.add_argument("--e2e-ncz", type=int, default=64,
                    help="rows per chunk of the end-to-end (host buffer) leg")
    ap.add_argument("--algorithm", default="fourierrec", choices=["fourierrec", "lprec", "linerec"])
    ap.add_argument("--filter", default="shepp")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-slab", type=int, default=512)
    ap.add_argument("--ref-rows", type=int, default=64)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", choices=["float32", "mixed"], default="float32",
                    help="path reported as value (the other one is timed beside it)")
    ap.add_argument("--no-mixed", action="store_true", help="time only --precision")
    ap.add_argument("--no-try", action="store_true", help="skip the try-centre sweep")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving stream")
    ap.add_argument("--serve-rate", type=float, default=50.0)
    ap.add_argument("--serve-requests", type=int, default=100)
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-ncz", type=int, default=16)
    ap.add_argument("--no-lamino", action="store_true", help="skip the laminography leg")
    ap.add_argument("--no-phase", action="store_true", help="skip the phase-retrieval leg")
    ap.add_argument("--phase-proj", type=int, default=64,
                    help="projections in the phase-retrieval leg")
    ap.add_argument("--ring-removal", action="store_true",
                    help="main leg with Fourier-wavelet ring removal (level 7, sigma 1, sym16)")
    ap.add_argument("--no-methods", action="store_true",
                    help="skip ring removal / lprec / linerec legs")
    ap.add_argument("--slab-rows", type=int, default=256,
                    help="rows of the lprec and linerec legs")
    ap.add_argument("--lam-n", type=int, default=1024)
    ap.add_argument("--lam-nproj", type=int, default=1200)
    ap.add_argument("--lam-rh", type=int, default=512)
    ap.add_argument("--try-n", type=int, default=4096)
    ap.add_argument("--try-nproj", type=int, default=3000)
    ap.add_argument("--try-centers", type=int, default=256)
    a = ap.parse_args()
    if a.warmup < 3:
        log("note: warmup < 3 requested; using 3")
        a.warmup = 3
    ws, rank, local = setup_dist()
    try:
        if a.impl == "reference":
            run_reference(a, ws, rank, local)
        else:
            run_ours(a, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
