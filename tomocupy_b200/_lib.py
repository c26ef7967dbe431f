"""ctypes binding of ``libtomocupy_b200.so`` (the C ABI in include/tomocupy_b200.h).

There is no fallback: if the CUDA library is missing or cannot be loaded,
importing an operator raises ``TcbLibraryError``.  Every C call returns a
status; a non-zero status is turned into ``TcbError`` carrying
``tcb_last_error()``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtomocupy_b200.so"

TCB_OK = 0
TCB_FLOAT32 = 0
TCB_FLOAT16 = 1
TCB_U8, TCB_U16, TCB_F32 = 0, 1, 2

PREP_DARKFLAT = 1
PREP_MINUS_LOG = 2
PREP_FLAT_LINEAR = 4
PREP_EDGE_PAD = 8

GRID_FP32 = 0
GRID_TENSOR = 1
GRID_TENSOR_FP32 = 2
GRID_TENSOR_STREAM = 3

TCF_OUT_ROWS = 0
TCF_OUT_PAIRS = 1

TCB_PHASE_PAGANIN = 0
TCB_PHASE_GPAGANIN = 1
TCB_PHASE_FARAGO = 2

FFF_OUT_ROWS = 0
FFF_OUT_PAIRS = 1
FFF_OUT_SPECTRUM = 2

TCB_ERR_OUT_OF_MEMORY = 4

STATUS_NAMES = {
    0: "TCB_OK", 1: "TCB_ERR_INVALID_ARGUMENT", 2: "TCB_ERR_CUDA", 3: "TCB_ERR_CUFFT",
    4: "TCB_ERR_OUT_OF_MEMORY", 5: "TCB_ERR_NOT_SUPPORTED", 6: "TCB_ERR_FREED",
}


class TcbLibraryError(RuntimeError):
    """The native library could not be loaded (not built, or no CUDA runtime)."""


class TcbError(RuntimeError):
    """A native call returned a non-zero tcb_status."""

    def __init__(self, status: int, func: str, msg: str):
        self.status = status
        super().__init__(f"{func} -> {STATUS_NAMES.get(status, status)}: {msg}")


vp, sz, f32, i32, u32, f64 = C.c_void_p, C.c_size_t, C.c_float, C.c_int, C.c_uint, C.c_double

# name -> argtypes (every function returns int)
SIGNATURES: dict[str, list] = {
    "tcb_version": [],
    "tcb_copy2d": [vp, sz, vp, sz, sz, sz, vp],
    "tcb_check_bounded_wait": [C.c_longlong, C.POINTER(i32), C.POINTER(C.c_longlong), vp],
    "tcb_profile_enable": [i32],
    "tcb_profile_report": [C.c_char_p, sz],
    "tcb_launch_count": [C.POINTER(C.c_uint64)],
    "tcb_darkflat_stats": [vp, vp, vp, vp, vp, sz, sz, sz, sz, i32, f32, i32, vp],
    "tcb_prep_rows": [vp, vp, vp, vp, vp, sz, sz, sz, sz, sz, i32, sz, sz, sz, sz, sz, u32, vp],
    "tcb_prep_noalloc": [vp, vp, vp, vp, sz, sz, sz, sz, sz, i32, f32, sz, sz, sz, sz, sz, u32,
                         vp],
    "tcb_stripe_fw_create": [C.POINTER(vp), sz, sz, sz, i32, f32, vp, vp, vp, vp, i32],
    "tcb_stripe_fw_apply_sino": [vp, vp, sz, vp],
    "tcb_stripe_fw_destroy": [vp],
    "tcb_filter_create": [C.POINTER(vp), sz, sz, sz, i32],
    "tcb_filter_apply": [vp, vp, vp, vp],
    "tcb_filter_destroy": [vp],
    "tcb_tcfilter_create": [C.POINTER(vp), sz, sz, sz, sz],
    "tcb_tcfilter_set_kernels": [vp, vp, sz, sz, vp],
    "tcb_tcfilter_apply": [vp, vp, vp, sz, sz, sz, vp, i32, sz, vp],
    "tcb_tcfilter_status": [vp, C.POINTER(i32)],
    "tcb_tcfilter_destroy": [vp],
    "tcb_fftfilter_create": [C.POINTER(vp), sz, sz, sz, sz],
    "tcb_fftfilter_set_kernels": [vp, vp, sz, sz, vp],
    "tcb_fftfilter_apply": [vp, vp, sz, sz, sz, sz, vp, i32, sz, vp],
    "tcb_fftfilter_destroy": [vp],
    "tcb_prep_rows_split16": [vp, vp, vp, vp, vp, vp, sz, sz, sz, sz, sz, i32, sz, sz, u32, vp],
    "tcb_downsample": [vp, vp, i32, sz, sz, sz, sz, sz, i32, vp],
    "tcb_pad360_weights": [vp, sz],
    "tcb_pad360_rows": [vp, sz, sz, sz, i32, vp, sz, vp],
    "tcb_rotate_proj": [vp, vp, sz, sz, sz, sz, sz, f64, f64, f64, f64, i32, vp],
    "tcb_dezinger": [vp, vp, i32, sz, sz, sz, sz, sz, i32, f64, vp],
    "tcb_stripe_ti_mask": [sz, f64, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "tcb_stripe_ti_create": [C.POINTER(vp), sz, sz, sz, f64, f64],
    "tcb_stripe_ti_apply_sino": [vp, vp, sz, sz, vp],
    "tcb_stripe_ti_destroy": [vp],
    "tcb_stripe_vo_create": [C.POINTER(vp), sz, sz, sz, f64, i32, i32, i32],
    "tcb_stripe_vo_apply": [vp, vp, sz, sz, vp],
    "tcb_stripe_vo_destroy": [vp],
    "tcb_phase_pads": [sz, sz, f64, f64, f64, i32, C.POINTER(sz), C.POINTER(sz)],
    "tcb_phase_create": [C.POINTER(vp), sz, sz, sz, i32, f64, f64, f64, f64, f64, f64, i32],
    "tcb_phase_sizes": [vp, C.POINTER(sz), C.POINTER(sz)],
    "tcb_phase_apply": [vp, vp, sz, vp],
    "tcb_phase_destroy": [vp],
    "tcb_fourierrec_create": [C.POINTER(vp), sz, sz, sz, vp, i32],
    "tcb_fourierrec_backprojection": [vp, vp, vp, vp],
    "tcb_fourierrec_backprojection_slices": [vp, vp, vp, vp],
    "tcb_fourierrec_pack": [vp, vp, vp, sz, sz, vp],
    "tcb_fourierrec_set_pairs_per_block": [vp, i32],
    "tcb_fourierrec_set_gridding": [vp, i32],
    "tcb_fourierrec_status": [vp, C.POINTER(i32)],
    "tcb_fourierrec_sample_positions": [vp, vp, vp, vp, vp, vp],
    "tcb_fourierrec_set_output": [vp, i32],
    "tcb_fourierrec_set_input_spectrum": [vp, i32],
    "tcb_fourierrec_destroy": [vp],
    "tcb_linerec_create": [C.POINTER(vp), sz, sz, sz, sz, sz, i32],
    "tcb_linerec_backprojection": [vp, vp, vp, vp, f32, i32, vp],
    "tcb_linerec_backprojection_try": [vp, vp, vp, vp, vp, f32, i32, vp],
    "tcb_linerec_backprojection_try_lamino": [vp, vp, vp, vp, vp, i32, vp],
    "tcb_linerec_status": [vp, C.POINTER(i32)],
    "tcb_linerec_destroy": [vp],
    "tcb_lprec_create": [C.POINTER(vp), sz, sz, sz, sz, sz, i32],
    "tcb_lprec_setgrids": [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, sz, sz],
    "tcb_lprec_backprojection": [vp, vp, vp, vp],
    "tcb_lprec_destroy": [vp],
    "tcb_fft2d_create": [C.POINTER(vp), sz, sz, sz],
    "tcb_fft2d_fwd": [vp, vp, vp, vp],
    "tcb_fft2d_destroy": [vp],
    "tcb_usfft2d_create": [C.POINTER(vp), sz, sz, sz, sz, sz, sz],
    "tcb_usfft2d_adj": [vp, vp, vp, vp, f32, i32, i32, vp],
    "tcb_usfft2d_adj_rows": [vp, vp, vp, vp, f32, i32, i32, i32, vp],
    "tcb_usfft2d_fwd": [vp, vp, vp, vp, f32, i32, i32, vp],
    "tcb_usfft2d_set_storage": [vp, i32, vp, vp],
    "tcb_usfft2d_sample_positions": [vp, vp, vp, vp, f32, i32, i32, vp],
    "tcb_usfft2d_destroy": [vp],
    "tcb_usfft1d_create": [C.POINTER(vp), sz, sz, sz, sz],
    "tcb_usfft1d_adj": [vp, vp, vp, f32, vp],
    "tcb_usfft1d_fwd": [vp, vp, vp, f32, vp],
    "tcb_usfft1d_set_storage": [vp, i32, vp],
    "tcb_usfft1d_destroy": [vp],
}

_lib = None


def load() -> C.CDLL:
    """Load the native library once; raise TcbLibraryError if unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("TOMOCUPY_B200_LIB", LIB_PATH))
    if not path.exists():
        raise TcbLibraryError(
            f"{path} not found: build it with `python -m tomocupy_b200.build` "
            "(the package has no CPU fallback)")
    try:
        lib = C.CDLL(str(path))
    except OSError as e:  # missing libcudart/libcufft on this machine
        raise TcbLibraryError(f"cannot load {path}: {e}") from e
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = C.c_int
    lib.tcb_last_error.argtypes = []
    lib.tcb_last_error.restype = C.c_char_p
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    """Call a C entry point and raise TcbError on a non-zero status."""
    lib = load()
    st = getattr(lib, name)(*args)
    if st != TCB_OK:
        msg = lib.tcb_last_error().decode(errors="replace")
        raise TcbError(st, name, msg)


def create(name: str, *args) -> C.c_void_p:
    """Call a *_create entry point and return the opaque handle."""
    h = C.c_void_p()
    call(name, C.byref(h), *args)
    return h


def ptr(x) -> int:
    """Device address of a torch tensor (or an int address passed through)."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    return x.data_ptr()


def stream_ptr(stream) -> int:
    """CUDA stream handle from a torch stream, a raw int, or None (current stream)."""
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    if hasattr(stream, "ptr"):
        return stream.ptr
    raise TypeError(f"cannot interpret {stream!r} as a CUDA stream")


def profile_enable(on: bool = True) -> None:
    """Start (clearing previous records) or stop per-stage CUDA-event timing."""
    call("tcb_profile_enable", int(on))


def profile_report() -> dict:
    """{stage: {"count": c, "ms": total, "bytes": b, "flops": f}} for the stages
    recorded since enable (b, f: the algorithmic bytes and FLOPs the stage's
    launches state, 0 where none is stated)."""
    import json
    buf = C.create_string_buffer(1 << 16)
    call("tcb_profile_report", buf, len(buf))
    return json.loads(buf.value.decode())


def launch_count() -> int:
    v = C.c_uint64(0)
    call("tcb_launch_count", C.byref(v))
    return int(v.value)
