"""Drive the reference's own CUDA operators (oracle/_ref/*.so) from torch.

The shared libraries are built by ``oracle/Makefile`` from the reference's
sources.  The classes below restate the reference's CuPy glue line by line
with torch tensors (GPU only), e.g. ``RefFourierRec.backprojection`` is
src/tomocupy/reconstruction/fourierrec.py:61-68.  Test infrastructure only.

Index arithmetic of the reference kernels is int32: callers keep
nz * (2n+2m)^2 (fourierrec) and nz * nproj * n below 2**31.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import torch

REF_DIR = Path(__file__).resolve().parent / "_ref"
_libs: dict = {}

vp, sz, f32, i32 = C.c_void_p, C.c_size_t, C.c_float, C.c_int

_SIGS = {
    "fourierrec": {"ref_create": ([sz, sz, sz, sz], vp), "ref_backprojection": ([vp, sz, sz, sz], None),
                   "ref_takexy": ([sz, sz, sz, sz, sz, sz], None)},
    "filter": {"ref_create": ([sz, sz, sz], vp), "ref_filter": ([vp, sz, sz, sz], None)},
    "linerec": {"ref_create": ([sz, sz, sz, sz, sz], vp),
                "ref_backprojection": ([vp, sz, sz, sz, f32, i32, sz], None),
                "ref_backprojection_try": ([vp, sz, sz, sz, sz, f32, i32, sz], None),
                "ref_backprojection_try_lamino": ([vp, sz, sz, sz, sz, i32, sz], None)},
    "lprec": {"ref_create": ([i32, i32, i32, i32, i32], vp),
              "ref_setgrids": ([vp] + [sz] * 13, None),
              "ref_backprojection": ([vp, sz, sz, sz], None)},
    "usfft1d": {"ref_create": ([sz, sz, sz, sz], vp), "ref_fwd": ([vp, sz, sz, f32, sz], None),
                "ref_adj": ([vp, sz, sz, f32, sz], None)},
    "usfft2d": {"ref_create": ([sz] * 6, vp), "ref_fwd": ([vp, sz, sz, sz, f32, i32, i32, sz], None),
                "ref_adj": ([vp, sz, sz, sz, f32, i32, i32, sz], None),
                "ref_take_x": ([sz, sz, sz, f32, i32, i32, i32, i32, i32, sz], None)},
    "fft2d": {"ref_create": ([sz, sz, sz], vp), "ref_fwd": ([vp, sz, sz, sz], None)},
}


def available() -> bool:
    return (REF_DIR / "libref_fourierrec.so").exists()


def lib(op: str, fp16: bool = False):
    key = (op, fp16)
    if key not in _libs:
        path = REF_DIR / f"libref_{op}{'_fp16' if fp16 else ''}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(str(path))
        for name, (args, res) in _SIGS[op].items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        L.ref_destroy.argtypes = [vp]
        L.ref_destroy.restype = None
        L.ref_last_error.argtypes = []
        L.ref_last_error.restype = C.c_int
        _libs[key] = L
    return _libs[key]


def _s(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


class _Handle:
    op = ""

    def __init__(self, fp16, *args):
        self.L = lib(self.op, fp16)
        self.h = self.L.ref_create(*args)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.ref_destroy(self.h)
                self.h = None
        except Exception:
            pass


class RefFourierRec(_Handle):
    """reconstruction/fourierrec.py:46-68 over the reference cfunc_fourierrec."""
    op = "fourierrec"

    def __init__(self, n, nproj, nz, theta, dtype="float32"):
        self.theta = theta.to(torch.float32).contiguous()
        self.nz, self.n, self.nproj = nz, n, nproj
        self.dtype = torch.float16 if dtype == "float16" else torch.float32
        super().__init__(dtype == "float16", nproj, nz // 2, n, self.theta.data_ptr())

    def backprojection(self, obj, data, stream=None):
        h = self.nz // 2
        data = torch.cat((data[:h, :, :, None], data[h:, :, :, None]), dim=3).reshape(
            data.shape).to(self.dtype).contiguous()
        assert obj.is_contiguous() and obj.dtype == self.dtype
        objc = obj.view(h, self.n, 2 * self.n)
        self.L.ref_backprojection(self.h, obj.data_ptr(), data.data_ptr(), _s(stream))
        obj[:] = torch.cat((objc[:, :, ::2], objc[:, :, 1::2]))
        return obj


class RefFilter(_Handle):
    """reconstruction/fbp_filter.py:45-58 over the reference cfunc_filter."""
    op = "filter"

    def __init__(self, n, ntheta, nz, dtype="float32"):
        self.dtype = torch.float16 if dtype == "float16" else torch.float32
        super().__init__(dtype == "float16", ntheta, nz, n)

    def filter(self, data, w, stream=None):
        assert data.is_contiguous()
        w = torch.view_as_real(w.contiguous()).to(self.dtype).contiguous()
        self.L.ref_filter(self.h, data.data_ptr(), w.data_ptr(), _s(stream))
        return data


def ref_fbp_filter_center(filt: RefFilter, data, wfilter, t, center, sht, n, ne):
    """backproj_functions.py:93-109 with torch standing in for CuPy."""
    nz = data.shape[0]
    pad = ne // 2 - n // 2
    tmp = torch.empty((nz, data.shape[1], ne), dtype=data.dtype, device=data.device)
    tmp[:, :, pad:pad + n] = data
    tmp[:, :, :pad] = data[:, :, :1]
    tmp[:, :, pad + n:] = data[:, :, -1:]
    if not torch.is_tensor(sht):
        sht = torch.full((nz,), float(sht), dtype=torch.float32, device=data.device)
    a = (-center + sht.reshape(-1).to(torch.float32)) + n / 2
    ci = float(torch.tensor(-2.0, dtype=torch.float32) * torch.tensor(math.pi, dtype=torch.float32))
    phase = (a * ci)[:, None] * t[None, :]
    w = torch.complex(wfilter * torch.cos(phase), wfilter * torch.sin(phase))
    filt.filter(tmp, w)
    data[:] = tmp[:, :, pad:pad + n]
    return data


class RefLineRec(_Handle):
    """reconstruction/linerec.py:44-85 over the reference cfunc_linerec."""
    op = "linerec"

    def __init__(self, theta, nproj, ncproj, nz, ncz, n, dtype="float32"):
        self.theta = theta.to(torch.float32).contiguous()
        super().__init__(dtype == "float16", nproj, nz, n, ncproj, ncz)

    def backprojection(self, f, data, stream=None, theta=None, lamino_angle=0.0, sz=0):
        if theta is None:
            theta = self.theta
            f[:] = 0
        phi = math.pi / 2 + lamino_angle / 180 * math.pi
        self.L.ref_backprojection(self.h, f.data_ptr(), data.contiguous().data_ptr(),
                                  theta.data_ptr(), phi, sz, _s(stream))

    def backprojection_try(self, f, data, sh, stream=None, theta=None, lamino_angle=0.0, sz=0):
        theta = self.theta if theta is None else theta
        phi = math.pi / 2 + lamino_angle / 180 * math.pi
        self.L.ref_backprojection_try(self.h, f.data_ptr(), data.contiguous().data_ptr(),
                                      theta.data_ptr(), sh.contiguous().data_ptr(), phi, sz,
                                      _s(stream))

    def backprojection_try_lamino(self, f, data, sh, stream=None, theta=None, lamino_angle=0.0,
                                  sz=0):
        theta = self.theta if theta is None else theta
        phi = (math.pi / 2 + (lamino_angle + sh.to(torch.float32)) / 180 * math.pi).contiguous()
        self.L.ref_backprojection_try_lamino(self.h, f.data_ptr(), data.contiguous().data_ptr(),
                                             theta.data_ptr(), phi.data_ptr(), sz, _s(stream))


class RefLpRec(_Handle):
    """reconstruction/lprec.py:292-335 over the reference cfunc_lprec.  ``grids``
    holds the Padj arrays (fZ, lp2p1, ..., cids) as NumPy arrays: the golden
    fixtures produced by the reference's own Python, or a restatement."""
    op = "lprec"

    def __init__(self, n, nproj, nz, grids, dtype="float32"):
        ntheta = 2 ** int(round(math.log2(nproj)))
        nrho = 2 * 2 ** int(round(math.log2(n)))
        super().__init__(dtype == "float16", nproj, nz, n, ntheta, nrho)
        import numpy as np
        dev = torch.device("cuda")
        tdt = torch.float16 if dtype == "float16" else torch.float32
        self.t = {}
        for k in ("lp2p1", "lp2p2", "lp2p1w", "lp2p2w", "C2lp1", "C2lp2", "lpids", "wids",
                  "cids"):
            self.t[k] = torch.as_tensor(np.ascontiguousarray(grids[k]), device=dev)
        fz = np.ascontiguousarray(grids["fZ"]).view("float32")
        self.t["fZ"] = torch.as_tensor(fz, device=dev).to(tdt).contiguous()
        t = self.t
        self.L.ref_setgrids(self.h, t["fZ"].data_ptr(), t["lp2p1"].data_ptr(),
                            t["lp2p2"].data_ptr(), t["lp2p1w"].data_ptr(), t["lp2p2w"].data_ptr(),
                            t["C2lp1"].data_ptr(), t["C2lp2"].data_ptr(), t["lpids"].data_ptr(),
                            t["wids"].data_ptr(), t["cids"].data_ptr(), len(grids["lpids"]),
                            len(grids["wids"]), len(grids["cids"]))

    def backprojection(self, obj, data, stream=None):
        data = data.contiguous()
        self.L.ref_backprojection(self.h, obj.data_ptr(), data.data_ptr(), _s(stream))
        return obj


def ref_darkflat_minus_log(data, dark, flat, bright_ratio=1.0, minus_log=True):
    """proc_functions.py:55-83 in torch, operation by operation (float32)."""
    dark0 = dark.to(torch.float32)
    flat0 = flat.to(torch.float32) / bright_ratio
    flat0 = flat0.mean(dim=0)
    dark0 = dark0.mean(dim=0)
    flat0 = flat0 * torch.tensor(1 + 1e-5, dtype=torch.float32)
    flat0 = flat0 - dark0
    res = (data.to(torch.float32) - dark0) / flat0
    if minus_log:
        res = torch.where(res <= 0, torch.ones((), dtype=torch.float32, device=res.device), res)
        res = -torch.log(res)
        res = torch.nan_to_num(res, nan=6.0, posinf=0.0, neginf=0.0)
    return res


# --------------------------------------------------------------------------
# laminography chain (reconstruction/lamfourierrec.py:46-73 and
# reconstruction/backproj_lamfourier_parallel.py:57-304, device-resident)
# --------------------------------------------------------------------------
class RefFFT2D(_Handle):
    op = "fft2d"

    def __init__(self, ntheta, detw, deth):
        super().__init__(False, ntheta, detw, deth)

    def fwd(self, g, f, stream=None):
        self.L.ref_fwd(self.h, g.data_ptr(), f.data_ptr(), _s(stream))


class RefUSFFT2D(_Handle):
    op = "usfft2d"

    def __init__(self, n0, n1, n2, ntheta, detw, deth):
        super().__init__(False, n0, n1, n2, ntheta, detw, deth)

    def adj(self, f, g, theta, phi, k, deth0, stream=None):
        self.L.ref_adj(self.h, f.data_ptr(), g.data_ptr(), theta.data_ptr(), phi, k, deth0,
                       _s(stream))

    def fwd(self, g, f, theta, phi, k, deth0, stream=None):
        self.L.ref_fwd(self.h, g.data_ptr(), f.data_ptr(), theta.data_ptr(), phi, k, deth0,
                       _s(stream))


class RefUSFFT1D(_Handle):
    op = "usfft1d"

    def __init__(self, n0, n1, n2, deth):
        super().__init__(False, n0, n1, n2, deth)

    def adj(self, f, g, phi, stream=None):
        self.L.ref_adj(self.h, f.data_ptr(), g.data_ptr(), phi, _s(stream))

    def fwd(self, g, f, phi, stream=None):
        self.L.ref_fwd(self.h, g.data_ptr(), f.data_ptr(), phi, _s(stream))


def ref_rec_lam(data, theta, center, lamino_angle, rh, wfilter, nthetac=8, dethc=8, n1c=8):
    """BackprojLamFourierParallel.rec_lam with the reference operators; the
    pinned host staging buffers become device tensors, the chunk packing and
    copies are restated with torch.  data: [ntheta, deth, detw] float32."""
    dev = data.device
    ntheta, deth, detw = data.shape
    n0, n1, n2 = rh, detw, detw
    ne = 4 * detw
    pad = ne // 2 - detw // 2
    t = (torch.arange(0, ne // 2 + 1, dtype=torch.float64, device=dev) / ne).to(torch.float32)
    phi = math.pi / 2 + lamino_angle / 180 * math.pi
    filt = RefFilter(ne, deth, nthetac)
    fft2 = RefFFT2D(nthetac, detw, deth)
    us2 = RefUSFFT2D(dethc, n1, n2, ntheta, detw, dethc)
    us1 = RefUSFFT1D(n0, n1c, n2, deth)
    th = theta.to(torch.float32).contiguous()
    # stage 1: filter rows of each projection, 2D FFT (fft2_chunks)
    s1 = torch.empty((ntheta, deth, detw // 2 + 1), dtype=torch.complex64, device=dev)
    ci = float(torch.tensor(-2.0, dtype=torch.float32) * torch.tensor(math.pi, dtype=torch.float32))
    for st in range(0, ntheta, nthetac):
        end = min(ntheta, st + nthetac)
        d0 = torch.zeros((nthetac, deth, detw), dtype=torch.float32, device=dev)
        d0[:end - st] = data[st:end]
        tmp = torch.empty((nthetac, deth, ne), dtype=torch.float32, device=dev)
        tmp[:, :, pad:pad + detw] = d0
        tmp[:, :, :pad] = d0[:, :, :1]
        tmp[:, :, pad + detw:] = d0[:, :, -1:]
        sht = torch.zeros((nthetac, 1), dtype=torch.float32, device=dev)
        a = -center + sht + n2 / 2                      # [nthetac, 1] float32
        phase = (t * ci)[None, :] * a                   # (c*t)*a order of the lamino glue
        w = torch.complex(wfilter * torch.cos(phase), wfilter * torch.sin(phase))
        filt.filter(tmp, w)
        d0 = tmp[:, :, pad:pad + detw].contiguous()
        g = torch.empty((nthetac, deth, detw // 2 + 1), dtype=torch.complex64, device=dev)
        fft2.fwd(g, d0)
        s1[st:end] = g[:end - st]
    # stage 2: usfft2d over chunks of frequency rows (usfft2d_chunks)
    nrow = deth // 2 + 1
    s2 = torch.empty((n1, nrow, n2), dtype=torch.complex64, device=dev)
    inp = torch.zeros((2 * ntheta, dethc, detw // 2 + 1), dtype=torch.complex64, device=dev)
    for k, st in enumerate(range(0, nrow, dethc)):
        end = min(nrow, st + dethc)
        s = end - st
        inp[:ntheta, :s] = s1[:, st:end]
        if k == 0:
            inp[ntheta:, dethc - s:dethc - 1] = s1[:, deth - end + 1:deth - st + 1]
            inp[ntheta:, dethc - 1] = s1[:, 0]
        else:
            inp[ntheta:, dethc - s:] = s1[:, deth - end + 1:deth - st + 1]
        out = torch.empty((n1, dethc, n2), dtype=torch.complex64, device=dev)
        us2.adj(out, inp, th, phi, k, deth)
        s2[:, st:end] = out[:, :s]
    # stage 3: usfft1d over chunks of rows (usfft1d_chunks)
    s3 = torch.empty((n1, n0, n2), dtype=torch.float32, device=dev)
    for st in range(0, n1, n1c):
        end = min(n1, st + n1c)
        gin = torch.zeros((n1c, nrow, n2), dtype=torch.complex64, device=dev)
        gin[:end - st] = s2[st:end]
        out = torch.empty((n1c, n0, n2), dtype=torch.float32, device=dev)
        us1.adj(out, gin, phi)
        s3[st:end] = out[:end - st]
    torch.cuda.synchronize()
    # stage 4: copyTransposed -> [rh, n1, n2]
    return s3.permute(1, 0, 2).contiguous()
