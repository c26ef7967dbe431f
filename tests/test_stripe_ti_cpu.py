"""Titarenko ring removal on the CPU: the NumPy restatement against
fixtures made by the reference's own remove_stripe_ti
(src/tomocupy/processing/remove_stripe.py:296-307, NumPy for CuPy), and the
library's host-side mask rule against Python's slice semantics."""
import ctypes as C
import sys

import numpy as np
import pytest

from conftest import ROOT


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import TI_CASES
    return TI_CASES


@pytest.mark.parametrize("i", range(4))
def test_oracle_matches_reference_fixture(i):
    from oracle import np_tomo
    nproj, nz, n, beta, mask, seed = _cases()[i]
    g = np.load(ROOT / "tests" / "golden" / "ti_stripe.npz")
    got = np_tomo.remove_stripe_ti(g[f"in_{i}"], beta, mask)
    assert np.array_equal(got, g[f"out_{i}"])


def test_mask_range_follows_python_slicing():
    from tomocupy_b200.processing.remove_stripe import ti_mask
    for n in (2, 48, 64, 100, 2048, 4096):
        for m in (0, 1, 2, 3, 0.25, 0.5, 0.75, 1.5, 0.333):
            ms = m * n
            sel = np.zeros(n, bool)
            sel[n // 2 - int(ms // 2):n // 2 + int(ms // 2)] = True
            a, b = ti_mask(n, m)
            want = np.flatnonzero(sel)
            got = np.arange(a, b)
            assert np.array_equal(got, want), (n, m, a, b)
