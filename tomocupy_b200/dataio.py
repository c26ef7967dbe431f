"""In-memory data sources and sinks for the reconstruction drivers.

The reference reads DXfile HDF5 files and writes tiff/h5/zarr
(src/tomocupy/dataio/reader.py, writer.py); file I/O is outside this
package.  ``ArrayReader`` holds the projection/dark/flat stacks in (ideally
pinned) host memory or on the device and derives every size exactly as the
reference reader does (``sizes.setup``).  ``ArrayWriter`` collects the
reconstructed slices into a host or device volume.
"""
from __future__ import annotations

import numpy as np
import torch

from . import sizes as _sizes
from .global_vars import args, params


def _as_tensor(x):
    if torch.is_tensor(x):
        return x
    return torch.from_numpy(np.ascontiguousarray(x))


def _binned(frames, b, slab=64):
    """float32 binning of [k, nz * 2^b, n * 2^b] frames on the GPU."""
    from .processing.proc_functions import downsample
    dev = frames.device if frames.is_cuda else torch.device("cuda")
    k, zr, nr = frames.shape
    nz, n = zr >> b, nr >> b
    out = torch.empty((k, nz, n), dtype=torch.float32, device=dev)
    for z0 in range(0, nz, slab):
        z1 = min(nz, z0 + slab)
        part = frames[:, z0 << b:z1 << b]
        if not part.is_cuda:
            part = part.to(dev)
        elif part.stride(2) != 1:
            part = part.contiguous()
        out[:, z0:z1] = downsample(part, b)
    return out


class ArrayReader:
    """Projections [nproj, nz, ni], darks [ndark, nz, ni], flats [nflat, nz, ni]."""

    def __init__(self, data, dark, flat, theta=None, pin=False):
        self.data = _as_tensor(data)
        self.dark = _as_tensor(dark)
        self.flat = _as_tensor(flat)
        if pin and self.data.device.type == "cpu":
            self.data = self.data.pin_memory()
            self.dark = self.dark.pin_memory()
            self.flat = self.flat.pin_memory()
        nproj, nz, ni = self.data.shape
        if theta is None:
            theta = _sizes.default_theta(nproj)
        self.theta_all = np.asarray(theta, dtype=np.float32)
        self.sizes = dict(nproji=nproj, nzi=nz, ni=ni, nflat=self.flat.shape[0],
                          ndark=self.dark.shape[0], dtype=str(self.data.dtype).split(".")[-1])
        _sizes.setup(self.sizes, self.theta_all, args, params)

    def frames(self):
        """(data, dark, flat) restricted to the selected projections and columns;
        with binning b > 0 the float32 2^b x 2^b block sums of those frames, as
        the reference's reader produces them (dataio/reader.py:335-356), on
        the GPU (host frames are binned slab by slab there)."""
        ids = params.ids_proj
        if isinstance(ids, (list, tuple)) and len(ids) == 2:
            sel = slice(ids[0], ids[1])
        else:
            sel = torch.as_tensor(np.asarray(ids))
        b = int(args.binning)
        c0 = args.start_column if args.dtype != "float16" else params.st_n
        c1 = c0 + params.ni * 2 ** b
        r0, r1 = args.start_row, args.start_row + params.nz * 2 ** b
        raw = (self.data[sel, r0:r1, c0:c1], self.dark[:, r0:r1, c0:c1],
               self.flat[:, r0:r1, c0:c1])
        if b == 0:
            return raw
        return tuple(_binned(t, b) for t in raw)


class ArrayWriter:
    """Collects slices into ``self.rec`` [nz, n, n] (host or device)."""

    def __init__(self, device="cpu", pin=False, dtype=torch.float32):
        self.device = torch.device(device)
        self.pin = pin
        self.dtype = dtype
        self.rec = None
        self.tries = {}

    def allocate(self, nz, n):
        if self.rec is None or self.rec.shape != (nz, n, n):
            rec = torch.empty((nz, n, n), dtype=self.dtype, device=self.device)
            if self.pin and self.device.type == "cpu":
                rec = rec.pin_memory()
            self.rec = rec
        return self.rec

    def write_data_chunk(self, rec, st, end, k):
        self.rec[st:end] = rec[:end - st]

    def write_data_try(self, rec, cid, id_slice):
        self.tries[(int(id_slice), float(cid))] = rec.detach().clone()
