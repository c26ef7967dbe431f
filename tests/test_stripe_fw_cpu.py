"""Fourier-wavelet ring removal on the CPU: the NumPy restatement
(oracle.np_tomo.remove_stripe_fw) against the fixtures made by the
reference's own remove_stripe_fw (src/tomocupy/processing/remove_stripe.py:51-293,
run with NumPy for CuPy by tests/golden/make_golden.py), bit for bit.

Both sides take their filter banks from tomocupy_b200.processing.wavelets
(PyWavelets is absent), so this pins the algorithm and its float32
operation order, not the published sym16/db5 tap tables."""
import sys

import numpy as np
import pytest

from conftest import ROOT


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import FW_CASES
    return FW_CASES


@pytest.mark.parametrize("i", range(4))
def test_oracle_matches_reference_fixture(i):
    from oracle import np_tomo
    from tomocupy_b200.processing import wavelets
    nproj, nz, n, level, sigma, wname, seed = _cases()[i]
    g = np.load(ROOT / "tests" / "golden" / "fw_stripe.npz")
    got = np_tomo.remove_stripe_fw(g[f"in_{i}"], sigma, level, wavelets.filter_bank(wname))
    want = g[f"out_{i}"]
    assert got.shape == want.shape
    assert np.array_equal(got, want), float(np.abs(got - want).max())
