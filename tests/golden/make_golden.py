"""Generate the golden fixtures in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py --cpu --ref <reference checkout>
    (or TOMOCUPY_REFERENCE in the environment)
        Executes the reference's own Python sources with NumPy standing in
        for CuPy (and stubs for h5py / the SWIG modules):
          * FBPFilter.calc_filter for every filter at several widths
            (src/tomocupy/reconstruction/fbp_filter.py:60-118)
          * Reader.init_sizes / init_sizes_try / init_sizes_lamino for a set
            of option combinations (src/tomocupy/dataio/reader.py:82-272)
          * paganin_filter / farago_filter (retrieve_phase.py:57-145)
        -> filter_spectra.npz, sizes_cases.json, ..., phase_retrieval.npz
          * remove_stripe_ti (remove_stripe.py:296-307) -> ti_stripe.npz
          * ProcFunctions.remove_outliers (proc_functions.py:96-107) -> dezinger.npz
          * ProcFunctions.pad360 (proc_functions.py:109-124) -> pad360.npz
          * utils.downsample (utils.py:157-167) -> downsample.npz
          * remove_all_stripe (remove_stripe.py:311-498) -> vo_stripe.npz
        (--phase / --ti / --dezinger / --pad360 / --downsample / --vo: only those)

    python tests/golden/make_golden.py --gpu --out DIR
        Runs the reference's CUDA operators (oracle/_ref, built from the
        reference sources) on small seeded inputs and stores their outputs
        -> ref_gpu_small.npz (needs a GPU; the inputs are re-generated from
        the stored seeds by the tests).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import types
from argparse import Namespace
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

FILTER_WIDTHS = (256, 1024, 2048, 4096)
FILTER_NAMES = ("none", "ramp", "shepp", "cosine", "cosine2", "hamming", "hann", "parzen")


def _numpy_as_cupy():
    cp = types.ModuleType("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cp, name, getattr(np, name))
    cp.fft = np.fft
    cp.linalg = np.linalg
    cp.asnumpy = np.asarray
    return cp


def _install_stubs():
    sys.modules["cupy"] = _numpy_as_cupy()
    pkg = types.ModuleType("tomocupy")
    pkg.__path__ = []
    sys.modules["tomocupy"] = pkg
    for sub in ("cfunc_filter", "cfunc_filterfp16", "utils"):
        m = types.ModuleType(f"tomocupy.{sub}")
        sys.modules[f"tomocupy.{sub}"] = m
        setattr(pkg, sub, m)
    import logging as _logging
    lg = types.ModuleType("tomocupy.logging")
    lg.getLogger = _logging.getLogger
    sys.modules["tomocupy.logging"] = lg
    pkg.logging = lg
    gv = types.ModuleType("tomocupy.global_vars")
    gv.args = Namespace()
    gv.params = Namespace()
    sys.modules["tomocupy.global_vars"] = gv
    pkg.global_vars = gv
    sys.modules["h5py"] = types.ModuleType("h5py")
    return gv


def _load(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


SIZE_CASES = [
    dict(sizes=dict(nproji=360, nzi=16, ni=512, nflat=10, ndark=10, dtype="uint16"), args={}),
    dict(sizes=dict(nproji=1500, nzi=2048, ni=2048, nflat=10, ndark=10, dtype="uint16"),
         args=dict(nsino_per_chunk=32)),
    dict(sizes=dict(nproji=1500, nzi=2048, ni=2448, nflat=20, ndark=10, dtype="uint16"),
         args=dict(dtype="float16")),
    dict(sizes=dict(nproji=721, nzi=100, ni=1001, nflat=10, ndark=5, dtype="uint16"),
         args=dict(start_column=3, end_column=-1, rotation_axis=480.5, nsino_per_chunk=1)),
    dict(sizes=dict(nproji=3000, nzi=1, ni=4096, nflat=10, ndark=10, dtype="uint16"),
         args=dict(reconstruction_type="try", rotation_axis=2048.0, center_search_width=48.0,
                   center_search_step=0.375, nsino="0")),
    dict(sizes=dict(nproji=1200, nzi=1024, ni=1024, nflat=10, ndark=10, dtype="uint16"),
         args=dict(lamino_angle=30.0, lamino_start_row=0, lamino_end_row=512,
                   reconstruction_type="full")),
    dict(sizes=dict(nproji=400, nzi=64, ni=256, nflat=10, ndark=10, dtype="uint16"),
         args=dict(reconstruction_type="try_lamino", lamino_angle=20.0,
                   lamino_search_width=2.0, lamino_search_step=0.5, nsino="[0.2,0.7]")),
    dict(sizes=dict(nproji=900, nzi=40, ni=640, nflat=10, ndark=10, dtype="uint16"),
         args=dict(start_proj=10, end_proj=890, blocked_views="[0.5,0.9]")),
]


def gen_cpu(ref: Path):
    gv = _install_stubs()
    fbp = _load(ref / "src/tomocupy/reconstruction/fbp_filter.py", "ref_fbp_filter")
    spectra = {}
    for ne in FILTER_WIDTHS:
        obj = fbp.FBPFilter.__new__(fbp.FBPFilter)
        obj.n = ne
        for name in FILTER_NAMES:
            spectra[f"{name}_{ne}"] = np.asarray(obj.calc_filter(name), dtype=np.float32)
    np.savez_compressed(HERE / "filter_spectra.npz", **spectra)

    reader = _load(ref / "src/tomocupy/dataio/reader.py", "ref_reader")
    from tomocupy_b200.config import DEFAULTS
    out = []
    for case in SIZE_CASES:
        args = Namespace(**DEFAULTS)
        for k, v in case["args"].items():
            setattr(args, k, v)
        gv.args.__dict__.clear()
        gv.args.__dict__.update(vars(args))
        gv.params.__dict__.clear()
        reader.args, reader.params = gv.args, gv.params
        r = reader.Reader.__new__(reader.Reader)
        sizes = case["sizes"]
        theta = np.linspace(0, np.pi, sizes["nproji"], dtype="float32")
        r.read_sizes = lambda s=sizes: dict(s)
        r.read_theta = lambda nproj, th=theta: th
        r.init_sizes()
        if gv.args.reconstruction_type[:3] == "try":
            r.init_sizes_try()
        if gv.args.lamino_angle != 0:
            r.init_sizes_lamino()
        p = {}
        for k, v in vars(gv.params).items():
            if isinstance(v, np.ndarray):
                p[k] = {"array": v.tolist(), "dtype": str(v.dtype)}
            elif isinstance(v, (np.integer,)):
                p[k] = int(v)
            elif isinstance(v, (np.floating,)):
                p[k] = float(v)
            elif isinstance(v, (list, tuple)):
                p[k] = [x.item() if hasattr(x, "item") else x for x in v]
            else:
                p[k] = v
        out.append({"case": case, "params": p,
                    "args_after": {k: getattr(gv.args, k) for k in
                                   ("end_row", "end_proj", "end_column")}})
    (HERE / "sizes_cases.json").write_text(json.dumps(out, indent=1, default=str))

    # log-polar grids of LpRec (lprec.py:82-289)
    sys.modules["cupy"]._default_memory_pool = types.SimpleNamespace(free_all_blocks=lambda: None)
    for sub in ("cfunc_lprec", "cfunc_lprecfp16"):
        m = types.ModuleType(f"tomocupy.{sub}")
        sys.modules[f"tomocupy.{sub}"] = m
        setattr(sys.modules["tomocupy"], sub, m)
    lp = _load(ref / "src/tomocupy/reconstruction/lprec.py", "ref_lprec")
    grids = {}
    for n, nproj in LPREC_CASES:
        ntheta = 2 ** int(np.round(np.log2(nproj)))
        nrho = 2 * 2 ** int(np.round(np.log2(n)))
        P = lp.create_gl(n, nproj, ntheta, nrho)
        A = lp.create_adj(P)
        for name in ("fZ", "lp2p1", "lp2p2", "lp2p1w", "lp2p2w", "C2lp1", "C2lp2", "cids",
                     "lpids", "wids"):
            grids[f"{name}_{n}_{nproj}"] = np.asarray(getattr(A, name))
    np.savez_compressed(HERE / "lprec_grids.npz", **grids)

    # Fourier-wavelet ring removal (remove_stripe.py:51-293).  PyWavelets is
    # absent: a stub serves the filter banks derived by
    # tomocupy_b200.processing.wavelets, so these fixtures pin the algorithm,
    # not the taps.
    from tomocupy_b200.processing import wavelets as W

    class _Wavelet:
        def __init__(self, name):
            self.dec_lo, self.dec_hi, self.rec_lo, self.rec_hi = (list(a) for a in
                                                                  W.filter_bank(name))
    pywt = types.ModuleType("pywt")
    pywt.Wavelet = _Wavelet
    pywt.dwt_coeff_len = lambda n, L, mode="symmetric": W.dwt_coeff_len(n, L)
    sys.modules["pywt"] = pywt
    import scipy.ndimage as ndi
    cx = types.ModuleType("cupyx")
    cxs = types.ModuleType("cupyx.scipy")
    cxn = types.ModuleType("cupyx.scipy.ndimage")
    for f in ("median_filter", "binary_dilation", "uniform_filter1d"):
        setattr(cxn, f, getattr(ndi, f))
    sys.modules.update({"cupyx": cx, "cupyx.scipy": cxs, "cupyx.scipy.ndimage": cxn})
    rs = _load(ref / "src/tomocupy/processing/remove_stripe.py", "ref_remove_stripe")
    fw = {}
    for i, (nproj, nz, n, level, sigma, wname, seed) in enumerate(FW_CASES):
        data = fw_input(nproj, nz, n, seed)
        fw[f"in_{i}"] = data
        fw[f"out_{i}"] = np.asarray(rs.remove_stripe_fw(data.copy(), sigma, wname, level),
                                    dtype=np.float32)
    np.savez_compressed(HERE / "fw_stripe.npz", **fw)
    print("wrote filter_spectra.npz, sizes_cases.json, lprec_grids.npz and fw_stripe.npz")
    gen_phase(ref)
    gen_ti(ref)
    gen_dezinger(ref)
    gen_pad360(ref)
    gen_downsample(ref)


# Phase retrieval (retrieve_phase.py:57-145): (method, nproj, dy, dz,
# pixel_size cm, dist cm, energy keV, alpha, delta/beta, W cm, seed).  The
# dist = 0 case on a power-of-two image and the 31-column farago case get a
# zero-wide edge padding on an axis, where the reference's prj[-0:] =
# prj[-1] gives every entry along that axis the last entry's value.
PHASE_CASES = [
    ("paganin", 3, 24, 40, 0.65e-4, 5.0, 20.0, 1e-3, 1500.0, 2e-4, 1),
    ("paganin", 2, 64, 96, 0.65e-4, 5.0, 20.0, 1e-3, 1500.0, 2e-4, 2),
    ("Gpaganin", 2, 24, 40, 0.65e-4, 5.0, 20.0, 1e-3, 1500.0, 1.3e-4, 3),
    ("farago", 2, 25, 30, 1e-4, 0.5, 25.0, 1e-3, 1000.0, 2e-4, 4),
    ("farago", 1, 20, 31, 1e-4, 0.5, 25.0, 1e-3, 1000.0, 2e-4, 6),
    ("paganin", 2, 16, 16, 1e-4, 0.0, 20.0, 1e-3, 1500.0, 2e-4, 5),
]


# Titarenko ring removal (remove_stripe.py:296-307): (nproj, nz, ni, beta,
# mask_size, seed).  Integer mask sizes only: the reference slices with
# mask_size * n, which NumPy and CuPy reject when it is a float; mask 2
# gives a negative slice start, i.e. the last n/2 columns.  Even widths
# only: for odd n the reference's irfft returns n - 1 samples and the add
# fails to broadcast.
TI_CASES = [
    (90, 4, 64, 0.022, 1, 1),
    (60, 3, 100, 0.05, 2, 2),
    (120, 2, 256, 0.022, 1, 3),
    (30, 2, 48, 0.022, 0, 4),
]


def ti_input(nproj, nz, ni, seed):
    """Seeded flat-normalised sinograms with column gain stripes."""
    rng = np.random.default_rng(seed)
    x = 0.7 + 0.1 * rng.random((nproj, nz, ni))
    gains = 1.0 + 0.03 * rng.standard_normal(ni) * (rng.random(ni) < 0.2)
    return (x * gains).astype(np.float32)


def gen_ti(ref: Path):
    """Runs remove_stripe_ti from the reference's own source with NumPy for
    CuPy -> ti_stripe.npz."""
    if "cupy" not in sys.modules:
        _install_stubs()
    for name in ("pywt", "cupyx", "cupyx.scipy", "cupyx.scipy.ndimage"):
        sys.modules.setdefault(name, types.ModuleType(name))
    nd = sys.modules["cupyx.scipy.ndimage"]
    for f in ("median_filter", "binary_dilation", "uniform_filter1d"):
        if not hasattr(nd, f):
            setattr(nd, f, None)
    rs = _load(ref / "src/tomocupy/processing/remove_stripe.py", "ref_remove_stripe_ti")
    out = {}
    for i, (nproj, nz, ni, beta, mask, seed) in enumerate(TI_CASES):
        data = ti_input(nproj, nz, ni, seed)
        out[f"in_{i}"] = data
        out[f"out_{i}"] = np.asarray(rs.remove_stripe_ti(data.copy(), beta, mask),
                                     dtype=np.float32)
    np.savez_compressed(HERE / "ti_stripe.npz", **out)
    print("wrote ti_stripe.npz")


# Vo's all-stripe removal, remove_all_stripe (remove_stripe.py:311-498):
# (nproj, nz, ni, snr, la_size, sm_size, seed).  Inputs have no repeated
# values inside a column (continuous noise; the dead column is constant up
# to 1e-6 noise), so every sort along the angles is unique: the fixtures do
# not depend on how an argsort orders ties (NumPy's default here, a stable
# sort in CuPy and in the library).
VO_CASES = [(90, 2, 64, 3.0, 21, 11, 1), (120, 3, 96, 3.0, 31, 11, 2),
            (64, 1, 80, 2.5, 11, 5, 3)]


def vo_input(nproj, nz, ni, seed):
    """Normalised sinogram-like data with partial, full and dead stripes,
    float32 [nproj, nz, ni], no ties along the angles."""
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, ni)
    ang = np.linspace(0, 1, nproj)[:, None, None]
    base = 0.6 + 0.3 * np.exp(-4 * (x[None, None, :] - 0.3 * np.sin(6 * ang)) ** 2)
    gain = 1 + 0.08 * rng.standard_normal(ni) * (rng.uniform(size=ni) < 0.15)
    data = base * gain[None, None, :] + 0.01 * rng.standard_normal((nproj, nz, ni))
    dead = rng.integers(4, ni - 4)
    data[:, :, dead] = 0.05 + 1e-6 * rng.standard_normal((nproj, nz))
    part = rng.integers(4, ni - 4)
    data[nproj // 3:, :, part] *= 1.15
    return data.astype(np.float32)


def gen_vo(ref: Path):
    """Runs remove_all_stripe from the reference's own source with NumPy for
    CuPy and scipy.ndimage for cupyx.scipy.ndimage -> vo_stripe.npz."""
    import scipy.ndimage as ndi
    if "cupy" not in sys.modules:
        _install_stubs()
    sys.modules.setdefault("pywt", types.ModuleType("pywt"))
    cx = types.ModuleType("cupyx")
    cxs = types.ModuleType("cupyx.scipy")
    cxn = types.ModuleType("cupyx.scipy.ndimage")
    for f in ("median_filter", "binary_dilation", "uniform_filter1d"):
        setattr(cxn, f, getattr(ndi, f))
    sys.modules.update({"cupyx": cx, "cupyx.scipy": cxs, "cupyx.scipy.ndimage": cxn})
    rs = _load(ref / "src/tomocupy/processing/remove_stripe.py", "ref_remove_stripe_vo")
    out = {}
    for i, (nproj, nz, ni, snr, la, sm, seed) in enumerate(VO_CASES):
        data = vo_input(nproj, nz, ni, seed)
        out[f"in_{i}"] = data
        out[f"out_{i}"] = np.asarray(rs.remove_all_stripe(data.copy(), snr, la, sm),
                                     dtype=np.float32)
    np.savez_compressed(HERE / "vo_stripe.npz", **out)
    print("wrote vo_stripe.npz")


# Outlier removal, ProcFunctions.remove_outliers (proc_functions.py:96-107):
# (dtype, nframes, nz, n, width, threshold, seed).  Widths 4 (an even window,
# upper median) and 5 on 3 frames (reflections beyond the first) included.
DEZINGER_CASES = [
    ("uint16", 20, 3, 40, 3, 500, 1),
    ("uint16", 12, 2, 33, 4, 300, 2),
    ("uint16", 10, 2, 64, 5, 1000, 3),
    ("uint16", 3, 2, 16, 5, 100, 4),
    ("float32", 15, 2, 30, 3, 0.05, 5),
]


# Binning, utils.downsample (utils.py:157-167) on float32 frames (the reader
# converts to float32 before binning): (nframes, rows, columns, binning,
# integer-valued, seed).
DOWNSAMPLE_CASES = [
    (3, 8, 16, 1, True, 1),
    (2, 8, 16, 2, False, 2),
    (2, 16, 24, 3, False, 3),
    (4, 6, 10, 1, False, 4),
]


def gen_downsample(ref: Path):
    """Runs utils.downsample from the reference's own source (NumPy for CuPy,
    a numexpr stand-in that evaluates 'x + y' with NumPy) -> downsample.npz."""
    import inspect
    if "cupy" not in sys.modules:
        _install_stubs()
    ne = types.ModuleType("numexpr")

    def evaluate(expr):
        f = inspect.currentframe().f_back
        return eval(expr, {}, dict(f.f_locals))
    ne.evaluate = evaluate
    sys.modules["numexpr"] = ne
    sys.modules.setdefault("tifffile", types.ModuleType("tifffile"))
    ut = _load(ref / "src/tomocupy/utils.py", "ref_utils")
    out = {}
    for i, (k, zr, nr, b, integer, seed) in enumerate(DOWNSAMPLE_CASES):
        rng = np.random.default_rng(seed)
        if integer:
            x = rng.integers(0, 65536, (k, zr, nr)).astype(np.float32)
        else:
            x = (rng.random((k, zr, nr)) * 1000).astype(np.float32)
        out[f"in_{i}"] = x
        out[f"out_{i}"] = np.asarray(ut.downsample(x, b), dtype=np.float32)
    np.savez_compressed(HERE / "downsample.npz", **out)
    print("wrote downsample.npz")


# Double-FOV padding, ProcFunctions.pad360 (proc_functions.py:109-124):
# (nproj, nz, ni, centeri, seed); center as Reader.init_sizes sets it for a
# double_fov scan (reader.py:143-149).
PAD360_CASES = [
    (5, 2, 64, 58.0, 1),     # axis on the right: no flip, w = 12
    (4, 3, 50, 6.5, 2),      # axis on the left: flip, w = 13
    (3, 1, 33, 30.25, 3),    # odd width, fractional centre
]


def gen_pad360(ref: Path):
    """Runs ProcFunctions.pad360 from the reference's own source with NumPy for
    CuPy -> pad360.npz."""
    if "cupy" not in sys.modules:
        _install_stubs()
    _proc_stubs()
    pf = _load(ref / "src/tomocupy/processing/proc_functions.py", "ref_proc_functions_360")
    gv = sys.modules["tomocupy.global_vars"]
    obj = pf.ProcFunctions.__new__(pf.ProcFunctions)
    out = {}
    for i, (nproj, nz, ni, centeri, seed) in enumerate(PAD360_CASES):
        rng = np.random.default_rng(seed)
        data = rng.random((nproj, nz, ni)).astype(np.float32)
        center = ni - centeri if centeri < ni // 2 else centeri
        gv.params.centeri, gv.params.ni, gv.params.center = centeri, ni, center
        pf.params = gv.params
        out[f"in_{i}"] = data
        out[f"out_{i}"] = np.asarray(obj.pad360(data.copy()), dtype=np.float32)
    np.savez_compressed(HERE / "pad360.npz", **out)
    print("wrote pad360.npz")


def _proc_stubs():
    """Modules that src/tomocupy/processing/proc_functions.py imports."""
    import scipy.ndimage as ndi
    sys.modules["cupy.fft"] = np.fft
    for name in ("cupyx", "cupyx.scipy"):
        sys.modules.setdefault(name, types.ModuleType(name))
    nd = types.ModuleType("cupyx.scipy.ndimage")
    nd.median_filter = ndi.median_filter
    sys.modules["cupyx.scipy.ndimage"] = nd
    sys.modules["cupyx.scipy"].ndimage = nd
    proc = types.ModuleType("tomocupy.processing")
    proc.__path__ = []
    proc.retrieve_phase = types.ModuleType("tomocupy.processing.retrieve_phase")
    proc.remove_stripe = types.ModuleType("tomocupy.processing.remove_stripe")
    sys.modules["tomocupy.processing"] = proc


def dezinger_input(dtype, nframes, nz, n, seed):
    """Seeded frames with sparse positive spikes (zingers)."""
    rng = np.random.default_rng(seed)
    if dtype == "uint16":
        x = rng.normal(10000, 300, (nframes, nz, n))
        x += (rng.random(x.shape) < 0.02) * rng.uniform(200, 20000, x.shape)
        return np.clip(x, 0, 65535).astype(np.uint16)
    x = rng.normal(0.7, 0.01, (nframes, nz, n))
    x += (rng.random(x.shape) < 0.02) * rng.uniform(0.01, 0.5, x.shape)
    return x.astype(np.float32)


def gen_dezinger(ref: Path):
    """Runs ProcFunctions.remove_outliers from the reference's own source with
    NumPy for CuPy and scipy.ndimage for cupyx.scipy.ndimage -> dezinger.npz."""
    if "cupy" not in sys.modules:
        _install_stubs()
    _proc_stubs()
    pf = _load(ref / "src/tomocupy/processing/proc_functions.py", "ref_proc_functions")
    gv = sys.modules["tomocupy.global_vars"]
    obj = pf.ProcFunctions.__new__(pf.ProcFunctions)
    out = {}
    for i, (dt, nf, nz, n, w, thr, seed) in enumerate(DEZINGER_CASES):
        data = dezinger_input(dt, nf, nz, n, seed)
        gv.args.dezinger, gv.args.dezinger_threshold = w, thr
        out[f"in_{i}"] = data
        out[f"out_{i}"] = np.asarray(obj.remove_outliers(data.copy()))
    np.savez_compressed(HERE / "dezinger.npz", **out)
    print("wrote dezinger.npz")


def phase_input(nproj, dy, dz, seed):
    """Seeded transmission-like projections in (0.2, 1): smooth field plus noise."""
    import scipy.ndimage as ndi
    rng = np.random.default_rng(seed)
    base = ndi.gaussian_filter(rng.standard_normal((nproj, dy, dz)), (0, 3, 3))
    base = base / (np.abs(base).max() + 1e-12)
    x = 0.6 + 0.3 * base + 0.02 * rng.standard_normal((nproj, dy, dz))
    return np.clip(x, 0.2, 1.0).astype(np.float32)


def gen_phase(ref: Path):
    """Runs paganin_filter / farago_filter from the reference's own source with
    NumPy for CuPy -> phase_retrieval.npz."""
    if "cupy" not in sys.modules:
        _install_stubs()
    sys.modules["cupy.fft"] = np.fft  # `from cupy.fft import fft2, ifft2`
    rp = _load(ref / "src/tomocupy/processing/retrieve_phase.py", "ref_retrieve_phase")
    out = {}
    for i, (meth, nproj, dy, dz, ps, dist, en, alpha, db, W, seed) in enumerate(PHASE_CASES):
        data = phase_input(nproj, dy, dz, seed)
        out[f"in_{i}"] = data
        if meth == "farago":
            res = rp.farago_filter(data.copy(), ps, dist, en, db, meth)
        else:
            res = rp.paganin_filter(data.copy(), ps, dist, en, alpha, meth, db, W)
        out[f"out_{i}"] = np.asarray(res, dtype=np.float32)
        py, pz, _ = rp._calc_pad(data, ps, dist, en, True)
        out[f"pads_{i}"] = np.array([py, pz], dtype=np.int64)
    np.savez_compressed(HERE / "phase_retrieval.npz", **out)
    print("wrote phase_retrieval.npz")


# (nproj, nz, ni, level, sigma, wavelet, seed)
FW_CASES = [(90, 2, 64, 3, 1.0, "sym16", 1), (120, 3, 96, 4, 2.0, "db5", 2),
            (64, 1, 80, 2, 1.0, "haar", 3), (100, 2, 128, 7, 1.0, "sym16", 4)]


def fw_input(nproj, nz, n, seed):
    """Normalised sinogram-like data with vertical stripes, float32 [nproj, nz, n]."""
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, n)
    base = np.exp(-4 * x ** 2)[None, None, :] * (1 + 0.1 * np.sin(
        np.linspace(0, 6, nproj))[:, None, None])
    stripes = 1 + 0.05 * rng.standard_normal(n) * (rng.uniform(size=n) < 0.2)
    noise = 0.01 * rng.standard_normal((nproj, nz, n))
    return (base * stripes[None, None, :] + noise).astype(np.float32)


LPREC_CASES = [(128, 90), (200, 128)]


GPU_CASES = dict(n=128, nproj=90, nz=4, seed=7)


def gpu_inputs():
    """Seeded inputs of the GPU golden cases (re-generated identically by the tests)."""
    import torch
    from tomocupy_b200 import synthetic
    c = GPU_CASES
    data, dark, flat, theta, _ = synthetic.make_dataset(c["nproj"], c["nz"], c["n"],
                                                        seed=c["seed"], device="cpu")
    return data, dark, flat, theta


def gen_gpu(out_dir: Path):
    import torch
    from oracle import refglue, np_tomo
    data, dark, flat, theta = gpu_inputs()
    c = GPU_CASES
    n, nproj, nz = c["n"], c["nproj"], c["nz"]
    dev = torch.device("cuda")
    d = torch.as_tensor(np_tomo.minus_log(np_tomo.darkflat(data.numpy(), dark.numpy(),
                                                           flat.numpy())))
    sino = d.permute(1, 0, 2).contiguous().to(dev)  # [nz, P, n]
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=dev)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=dev)
    filt = refglue.RefFilter(ne, nproj, nz)
    filtered = refglue.ref_fbp_filter_center(filt, sino.clone(), wf, t, n / 2, 0.0, n, ne)
    th = torch.as_tensor(theta, device=dev)
    fr = refglue.RefFourierRec(n, nproj, nz, th)
    rec_fr = torch.zeros((nz, n, n), dtype=torch.float32, device=dev)
    fr.backprojection(rec_fr, filtered.clone())
    lr = refglue.RefLineRec(th, nproj, nproj, nz, nz, n)
    rec_lr = torch.zeros((nz, n, n), dtype=torch.float32, device=dev)
    lr.backprojection(rec_lr, filtered.clone())
    torch.cuda.synchronize()
    out_dir.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out_dir / "ref_gpu_small.npz", filtered=filtered.cpu().numpy(),
                        fourierrec=rec_fr.cpu().numpy(), linerec=rec_lr.cpu().numpy(),
                        **{k: np.int64(v) for k, v in GPU_CASES.items()})
    print("wrote", out_dir / "ref_gpu_small.npz")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--phase", action="store_true", help="only phase_retrieval.npz")
    ap.add_argument("--ti", action="store_true", help="only ti_stripe.npz")
    ap.add_argument("--dezinger", action="store_true", help="only dezinger.npz")
    ap.add_argument("--pad360", action="store_true", help="only pad360.npz")
    ap.add_argument("--downsample", action="store_true", help="only downsample.npz")
    ap.add_argument("--vo", action="store_true", help="only vo_stripe.npz")
    ap.add_argument("--ref", default=os.environ.get("TOMOCUPY_REFERENCE"),
                    required="TOMOCUPY_REFERENCE" not in os.environ)
    ap.add_argument("--out", default=str(HERE))
    a = ap.parse_args()
    if a.cpu:
        gen_cpu(Path(a.ref))
    else:
        if a.phase:
            gen_phase(Path(a.ref))
        if a.ti:
            gen_ti(Path(a.ref))
        if a.dezinger:
            gen_dezinger(Path(a.ref))
        if a.pad360:
            gen_pad360(Path(a.ref))
        if a.downsample:
            gen_downsample(Path(a.ref))
        if a.vo:
            gen_vo(Path(a.ref))
    if a.gpu:
        gen_gpu(Path(a.out))
