"""The C-ABI library loads without a GPU and exports every symbol the header declares."""
import ctypes
import re

from conftest import ROOT


def header_functions():
    text = (ROOT / "include" / "tomocupy_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tcb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = header_functions()
    assert "tcb_fourierrec_backprojection" in names
    assert "tcb_filter_apply" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from tomocupy_b200 import _lib
    lib = _lib.load()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert lib.tcb_version() >= 100


def test_binding_signatures_cover_header():
    from tomocupy_b200 import _lib
    declared = set(header_functions()) - {"tcb_last_error"}
    bound = set(_lib.SIGNATURES)
    assert declared == bound, (declared - bound, bound - declared)


def test_invalid_arguments_raise_without_gpu():
    """Argument validation happens on the host before any CUDA call."""
    import pytest
    from tomocupy_b200 import _lib
    with pytest.raises(_lib.TcbError) as e:
        _lib.create("tcb_fourierrec_create", 10, 1, 7, 0, 0)  # null theta
    assert e.value.status == 1
    with pytest.raises(_lib.TcbError):
        _lib.create("tcb_filter_create", 10, 1, 7, 0)  # odd n
    with pytest.raises(_lib.TcbError):
        _lib.create("tcb_linerec_create", 10, 1, 64, 10, 1, 5)  # bad precision
    h = ctypes.c_void_p(0)
    with pytest.raises(_lib.TcbError):
        _lib.call("tcb_fourierrec_backprojection", h, 0, 0, 0)
