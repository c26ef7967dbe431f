"""Drop-in for ``tomocupy.cfunc_lprecfp16``: fp16 buffers, fp32 arithmetic inside."""
from . import _lib
from .cfunc_lprec import cfunc_lprec as _fp32


class cfunc_lprec(_fp32):
    _precision = _lib.TCB_FLOAT16
