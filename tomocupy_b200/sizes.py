"""Size, centre and chunk bookkeeping of the reference reader.

Restates ``Reader.init_sizes`` / ``init_sizes_try`` / ``init_sizes_lamino``
(src/tomocupy/dataio/reader.py:82-272) on plain shapes instead of an HDF5
file, so the chunking, the even-width trim, binning, the float16
power-of-two crop, the try-centre shift list and the laminography height
are bit-identical to the reference's.
"""
from __future__ import annotations

from ast import literal_eval

import numpy as np


def default_theta(nproj: int) -> np.ndarray:
    """Angles used when a file has no /exchange/theta (reader.py:317)."""
    return np.linspace(0, np.pi, nproj, dtype="float32")


def init_sizes(sizes: dict, theta: np.ndarray, args, params, log=None) -> None:
    """Fill ``params`` from the data sizes; may adjust ``args.end_*`` like the reference."""
    nproji = sizes["nproji"]
    nzi = sizes["nzi"]
    ni = sizes["ni"]
    nflat = sizes["nflat"]
    ndark = sizes["ndark"]
    dtype = sizes["dtype"]

    in_dtype = args.dtype if args.binning > 0 else dtype

    if args.end_row == -1:
        args.end_row = nzi
    if args.end_proj == -1:
        args.end_proj = nproji
    if args.end_column == -1:
        args.end_column = ni

    nz = args.end_row - args.start_row

    ncz = args.nsino_per_chunk
    if ncz == 1 and args.reconstruction_algorithm == "fourierrec":
        ncz = 2  # two rows travel as one complex sinogram

    ncproj = args.nproj_per_chunk

    centeri = args.rotation_axis
    if centeri == -1:
        centeri = ni / 2

    st_n = args.start_column
    end_n = args.end_column

    # work only with multiples of 2
    nsh = (end_n - st_n) % (2 ** (args.binning + 1))
    if nsh != 0:
        end_n -= nsh
        if log:
            log.warning(f"Decreasing projection width by {nsh} pixel. "
                        f"New projection width: {end_n - st_n}")

    ni = end_n - st_n
    centeri -= st_n

    ni //= 2 ** args.binning
    centeri /= 2 ** args.binning
    nz //= 2 ** args.binning

    if args.file_type == "double_fov":
        n = 2 * ni
        center = ni - centeri if centeri < ni // 2 else centeri
    else:
        n = ni
        center = centeri

    if args.dtype == "float16":
        center += (2 ** int(np.log2(ni)) - ni) / 2
        st_n = (ni - 2 ** int(np.log2(ni))) // 2
        end_n = st_n + 2 ** int(np.log2(ni))
        ni = 2 ** int(np.log2(ni))
        n = 2 ** int(np.log2(n))

    ids_proj = [args.start_proj, args.end_proj]
    theta = np.asarray(theta)[ids_proj[0]:ids_proj[1]]
    if args.blocked_views != "none":
        tmp = literal_eval(args.blocked_views)
        if not isinstance(tmp[0], list):
            tmp = [tmp]
        ids = np.arange(len(theta))
        for pairs in tmp:
            [st, end] = pairs
            ids = np.intersect1d(ids, np.where(((theta) % np.pi < st) +
                                               ((theta - st) % np.pi > end - st))[0])
        theta = theta[ids]
        ids_proj = np.arange(ids_proj[0], ids_proj[1])[ids]
    nproj = len(theta)

    nzchunk = int(np.ceil(nz / ncz))
    lzchunk = np.minimum(ncz, np.int32(nz - np.arange(nzchunk) * ncz))
    ntchunk = int(np.ceil(nproj / ncproj))
    ltchunk = np.minimum(ncproj, np.int32(nproj - np.arange(ntchunk) * ncproj))

    tmp = literal_eval(args.nsino)
    if not isinstance(tmp, list):
        tmp = [tmp]

    params.id_slices = np.int32(np.array(tmp) * (nz * 2 ** args.binning - 1) /
                                2 ** args.binning) * 2 ** args.binning
    params.n = n
    params.nz = nz
    params.ncz = ncz
    params.nproj = nproj
    params.ncproj = ncproj
    params.center = center
    params.ni = ni
    params.nzi = nzi
    params.centeri = centeri
    params.ndark = ndark
    params.nflat = nflat
    params.ids_proj = ids_proj
    params.theta = theta
    params.nzchunk = nzchunk
    params.lzchunk = lzchunk
    params.ntchunk = ntchunk
    params.ltchunk = ltchunk
    params.dtype = args.dtype
    params.in_dtype = in_dtype
    params.st_n = st_n
    params.end_n = end_n
    params.shape_data_full = (nproj, nz, ni)
    params.shape_data_fulln = (nproj, nz, n)


def init_sizes_try(args, params) -> None:
    """Centre (or tilt) sweep list and its chunking (reader.py:224-247)."""
    if args.reconstruction_type == "try":
        shift_array = np.arange(-args.center_search_width, args.center_search_width,
                                args.center_search_step * 2 ** args.binning
                                ).astype("float32") / 2 ** args.binning
        save_centers = (params.centeri - shift_array) * 2 ** args.binning + params.st_n
        if (args.file_type == "double_fov") and (params.centeri < params.ni // 2):
            shift_array = -shift_array
    elif args.reconstruction_type == "try_lamino":
        shift_array = np.arange(-args.lamino_search_width, args.lamino_search_width,
                                args.lamino_search_step).astype("float32")
        save_centers = args.lamino_angle + shift_array
    else:
        raise ValueError(f"init_sizes_try: reconstruction_type={args.reconstruction_type!r}")
    nschunk = int(np.ceil(len(shift_array) / params.ncz))
    lschunk = np.minimum(params.ncz, np.int32(len(shift_array) - np.arange(nschunk) * params.ncz))
    params.shift_array = shift_array
    params.save_centers = save_centers
    params.nschunk = nschunk
    params.lschunk = lschunk


def init_sizes_lamino(args, params) -> None:
    """Laminography reconstruction height and row chunks (reader.py:249-272)."""
    rh0 = int(np.ceil((params.nz * 2 ** args.binning / np.cos(args.lamino_angle / 180 * np.pi)
                       ) / 2 ** args.binning / 2)) * 2
    if args.lamino_end_row == -1:
        rh = rh0
    else:
        rh = args.lamino_end_row // 2 ** args.binning - args.lamino_start_row // 2 ** args.binning
    nrchunk = int(np.ceil(rh / params.ncz))
    lrchunk = np.minimum(params.ncz, np.int32(rh - np.arange(nrchunk) * params.ncz))
    params.nrchunk = nrchunk
    params.lrchunk = lrchunk
    params.rh = rh
    params.lamino_angle = args.lamino_angle
    params.lamino_start_row = args.lamino_start_row // 2 ** args.binning
    params.lamino_shift = (rh0 // 2 - rh // 2) - args.lamino_start_row // 2 ** args.binning


def setup(sizes: dict, theta, args, params, log=None) -> None:
    """Everything the reference Reader.__init__ computes (reader.py:64-80)."""
    init_sizes(sizes, theta, args, params, log)
    if args.reconstruction_type[:3] == "try":
        init_sizes_try(args, params)
    if args.lamino_angle != 0:
        init_sizes_lamino(args, params)
