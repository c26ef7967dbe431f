"""Double-FOV padding on the CPU: the NumPy restatement against fixtures made
by the reference's own ProcFunctions.pad360
(src/tomocupy/processing/proc_functions.py:109-124, NumPy for CuPy), and the
library's host-side transition weights against NumPy's float64 formula."""
import ctypes as C
import sys

import numpy as np
import pytest

from conftest import ROOT


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import PAD360_CASES
    return PAD360_CASES


@pytest.mark.parametrize("i", range(3))
def test_oracle_matches_reference_fixture(i):
    from oracle import np_tomo
    nproj, nz, ni, centeri, seed = _cases()[i]
    center = ni - centeri if centeri < ni // 2 else centeri
    g = np.load(ROOT / "tests" / "golden" / "pad360.npz")
    assert np.array_equal(np_tomo.pad360(g[f"in_{i}"], centeri, ni, center), g[f"out_{i}"])


@pytest.mark.parametrize("w", [1, 2, 13, 100, 1023])
def test_transition_weights_match_numpy(w):
    """Same float64 steps; the integer powers come from libm's pow here and
    from NumPy's own power loops (CuPy's device pow in the reference), which
    may differ in the last bit; the polynomial's cancellation near v = 1 (its
    terms sum to 1 from magnitudes up to 540) turns that into ~1e-13
    relative, still far below the float32 rounding of the product the
    weights feed."""
    from tomocupy_b200 import _lib
    v = np.empty(w, dtype=np.float64)
    _lib.call("tcb_pad360_weights", v.ctypes.data_as(C.c_void_p), w)
    x = np.linspace(1, 0, w, endpoint=False)
    want = x ** 5 * (126 - 420 * x + 540 * x ** 2 - 315 * x ** 3 + 70 * x ** 4)
    assert np.allclose(v, want, rtol=1e-12, atol=1e-300)
