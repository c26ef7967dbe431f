"""Vo's all-stripe removal on the CPU: the NumPy restatement
(oracle.np_tomo.remove_all_stripe) against fixtures made by the reference's
own remove_all_stripe (src/tomocupy/processing/remove_stripe.py:311-498, run
with NumPy for CuPy and scipy.ndimage for cupyx.scipy.ndimage by
tests/golden/make_golden.py --vo), bit for bit.  The restatement keeps the
reference's array layouts, so its float32 reductions add in the same order."""
import sys

import numpy as np
import pytest

from conftest import ROOT


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import VO_CASES
    return VO_CASES


@pytest.mark.parametrize("i", range(3))
def test_oracle_matches_reference_fixture(i):
    from oracle import np_tomo
    nproj, nz, ni, snr, la, sm, seed = _cases()[i]
    g = np.load(ROOT / "tests" / "golden" / "vo_stripe.npz")
    got = np_tomo.remove_all_stripe(g[f"in_{i}"], snr, la, sm)
    assert np.array_equal(got, g[f"out_{i}"])
