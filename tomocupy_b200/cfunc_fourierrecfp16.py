"""Drop-in for ``tomocupy.cfunc_fourierrecfp16``: fp16 buffers, fp32 arithmetic inside."""
from . import _lib
from .cfunc_fourierrec import cfunc_fourierrec as _fp32


class cfunc_fourierrec(_fp32):
    _precision = _lib.TCB_FLOAT16
