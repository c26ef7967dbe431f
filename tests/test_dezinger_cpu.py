"""Outlier removal on the CPU: the NumPy/SciPy restatement against fixtures
made by the reference's own ProcFunctions.remove_outliers
(src/tomocupy/processing/proc_functions.py:96-107, NumPy for CuPy and
scipy.ndimage for cupyx.scipy.ndimage)."""
import sys

import numpy as np
import pytest

from conftest import ROOT


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import DEZINGER_CASES
    return DEZINGER_CASES


@pytest.mark.parametrize("i", range(5))
def test_oracle_matches_reference_fixture(i):
    from oracle import np_tomo
    dt, nf, nz, n, w, thr, seed = _cases()[i]
    g = np.load(ROOT / "tests" / "golden" / "dezinger.npz")
    got = np_tomo.dezinger(g[f"in_{i}"], w, thr)
    assert got.dtype == g[f"out_{i}"].dtype
    assert np.array_equal(got, g[f"out_{i}"])
