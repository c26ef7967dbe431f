"""Drop-in for the reference module ``tomocupy.cfunc_fourierrec``.

Same class name, constructor argument order and method signature as the SWIG
class (src/cuda/cfunc_fourierrec.i:9-21): pointers and streams are integer
addresses.  ``nz`` counts complex slice pairs; ``g`` is overwritten during
``backprojection`` exactly as in the reference.
"""
from __future__ import annotations

from . import _lib


class cfunc_fourierrec:
    _precision = _lib.TCB_FLOAT32

    def __init__(self, nproj, nz, n, theta_):
        self._h = _lib.create("tcb_fourierrec_create", int(nproj), int(nz), int(n),
                              _lib.ptr(theta_), self._precision)
        self._n, self._nproj, self._nz = int(n), int(nproj), int(nz)

    # read-only attributes, as %immutable in the SWIG interface
    n = property(lambda self: self._n)
    nproj = property(lambda self: self._nproj)
    nz = property(lambda self: self._nz)

    def backprojection(self, f, g, stream):
        """f complex [nz, n, n] <- backprojection of g complex [nz, nproj, n]."""
        self._check()
        _lib.call("tcb_fourierrec_backprojection", self._h, _lib.ptr(f), _lib.ptr(g),
                  _lib.stream_ptr(stream))

    def backprojection_slices(self, f, g, stream):
        """f real [2*nz, n, n] (pair k -> slices k and nz+k) from g complex [nz, nproj, n]."""
        self._check()
        _lib.call("tcb_fourierrec_backprojection_slices", self._h, _lib.ptr(f), _lib.ptr(g),
                  _lib.stream_ptr(stream))

    def pack(self, g, src, row_stride, xoff, stream):
        """g[k] = src[k, :, xoff:xoff+n] + 1j*src[k+nz, :, xoff:xoff+n]."""
        self._check()
        _lib.call("tcb_fourierrec_pack", self._h, _lib.ptr(g), _lib.ptr(src), int(row_stride),
                  int(xoff), _lib.stream_ptr(stream))

    def set_pairs_per_block(self, pairs: int) -> None:
        """Tuning knob (not in the reference): slice pairs per gridding block, 0 = auto."""
        self._check()
        _lib.call("tcb_fourierrec_set_pairs_per_block", self._h, int(pairs))

    def set_gridding(self, mode: int) -> None:
        """_lib.GRID_FP32 (default, the drop-in) or _lib.GRID_TENSOR (mixed precision)."""
        self._check()
        _lib.call("tcb_fourierrec_set_gridding", self._h, int(mode))

    def set_output(self, precision: int) -> None:
        """_lib.TCB_FLOAT16: fp16 output slices from fp32 input (not in the reference)."""
        self._check()
        _lib.call("tcb_fourierrec_set_output", self._h, int(precision))

    def set_input_spectrum(self, on: bool) -> None:
        """g holds the projection FFT already (FFTFilter spectrum output; not in the reference)."""
        self._check()
        _lib.call("tcb_fourierrec_set_input_spectrum", self._h, int(bool(on)))

    def sample_positions(self):
        """(x, y, fx, fy) [nproj, n]: the polar sample coordinates (takexy's) and
        the floor(2n x), floor(2n y) that place the footprints, as the gridding
        kernels compute them (a test hook; not in the reference)."""
        import torch
        self._check()
        dev = torch.device("cuda", torch.cuda.current_device())
        x = torch.empty((self._nproj, self._n), dtype=torch.float32, device=dev)
        y = torch.empty_like(x)
        fx = torch.empty((self._nproj, self._n), dtype=torch.int32, device=dev)
        fy = torch.empty_like(fx)
        _lib.call("tcb_fourierrec_sample_positions", self._h, x.data_ptr(), y.data_ptr(),
                  fx.data_ptr(), fy.data_ptr(), _lib.stream_ptr(None))
        return x, y, fx, fy

    def timed_out(self) -> bool:
        """True when a tensor-core gridding wait gave up (synchronises)."""
        import ctypes as C
        self._check()
        v = C.c_int(0)
        _lib.call("tcb_fourierrec_status", self._h, C.byref(v))
        return bool(v.value)

    def _check(self):
        if self._h is None:
            raise _lib.TcbError(6, type(self).__name__, "object was freed")

    def free(self):
        """Release device memory; idempotent like the reference's is_free guard."""
        if getattr(self, "_h", None) is not None:
            _lib.call("tcb_fourierrec_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
