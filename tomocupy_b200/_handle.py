"""Common lifetime handling of the native operator handles."""
from __future__ import annotations

from . import _lib


class NativeHandle:
    """Owns one C handle; ``free()`` is idempotent like the reference's ``is_free``."""

    _destroy = ""

    def _set(self, h):
        self._h = h

    def _live(self):
        h = getattr(self, "_h", None)
        if h is None:
            raise _lib.TcbError(6, type(self).__name__, "object was freed")
        return h

    def free(self):
        if getattr(self, "_h", None) is not None:
            _lib.call(self._destroy, self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
