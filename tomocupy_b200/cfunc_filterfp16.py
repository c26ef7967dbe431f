"""Drop-in for ``tomocupy.cfunc_filterfp16``: fp16 buffers, fp32 transforms inside."""
from . import _lib
from .cfunc_filter import cfunc_filter as _fp32


class cfunc_filter(_fp32):
    _precision = _lib.TCB_FLOAT16
