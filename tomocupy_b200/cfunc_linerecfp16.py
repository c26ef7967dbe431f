"""Drop-in for ``tomocupy.cfunc_linerecfp16``: fp16 buffers, fp32 accumulation inside."""
from . import _lib
from .cfunc_linerec import cfunc_linerec as _fp32


class cfunc_linerec(_fp32):
    _precision = _lib.TCB_FLOAT16
