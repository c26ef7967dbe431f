"""Binning on the CPU: the NumPy restatement against fixtures made by the
reference's own utils.downsample (src/tomocupy/utils.py:157-167)."""
import sys

import numpy as np
import pytest

from conftest import ROOT


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import DOWNSAMPLE_CASES
    return DOWNSAMPLE_CASES


@pytest.mark.parametrize("i", range(4))
def test_oracle_matches_reference_fixture(i):
    from oracle import np_tomo
    k, zr, nr, b, integer, seed = _cases()[i]
    g = np.load(ROOT / "tests" / "golden" / "downsample.npz")
    assert np.array_equal(np_tomo.downsample(g[f"in_{i}"], b), g[f"out_{i}"])
