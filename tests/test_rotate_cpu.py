"""CPU checks of the projection-rotation oracle: pinned against
scipy.ndimage.rotate (the published implementation whose semantics cupyx's
rotate, called by the reference's rotate_proj, follows), and the host-side
parameters against the oracle's."""
import numpy as np
import pytest
import scipy
from scipy import ndimage, special

from oracle import np_tomo


def _scipy_params(angle, nz, n):
    # scipy forms its matrix with cosdg/sindg; the rest is the same
    c, s = float(special.cosdg(angle)), float(special.sindg(angle))
    rot = np.array([[c, s], [-s, c]])
    shape = np.array([nz, n], dtype=np.float64)
    off = (shape - 1) / 2 - rot @ ((shape - 1) / 2)
    return c, s, float(off[0]), float(off[1])


@pytest.mark.parametrize("angle", [0.7, -2.25, 15.0, 90.0, 181.3])
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("shape", [(3, 17, 40), (2, 32, 31), (1, 1, 9)])
def test_rotate_oracle_matches_scipy(angle, order, shape):
    rng = np.random.default_rng(11)
    data = rng.random(shape, dtype=np.float32) * 3 - 1
    want = ndimage.rotate(data, angle, reshape=False, order=order, axes=(2, 1),
                          mode="nearest")
    got = np_tomo.rotate_planes(data, *_scipy_params(angle, shape[1], shape[2]), order=order)
    assert got.dtype == np.float32 and got.shape == want.shape
    # same matrix and offsets: the restatement reproduces scipy bit for bit
    assert np.array_equal(got, want), (scipy.__version__, np.abs(got - want).max())


@pytest.mark.parametrize("angle", [0.7, -2.25, 15.0])
def test_rotate_oracle_numpy_trig_within_ulp_of_scipy(angle):
    """With NumPy's cos/sin (the reference's host arithmetic) instead of
    scipy's cosdg/sindg, results stay within a float32 ulp or two."""
    rng = np.random.default_rng(12)
    data = rng.random((2, 24, 48), dtype=np.float32)
    want = ndimage.rotate(data, angle, reshape=False, order=1, axes=(2, 1), mode="nearest")
    got = np_tomo.rotate_proj(data, angle, order=1)
    assert np.all(np.abs(got - want) <= 2 * np.spacing(np.abs(want)) + 1e-12)


def test_rotate_params_host_matches_oracle():
    from tomocupy_b200.processing.proc_functions import rotate_params
    for angle, nz, n in [(0.7, 17, 40), (-3.5, 2048, 2448), (33.0, 1, 5)]:
        assert rotate_params(angle, nz, n) == np_tomo.rotate_params(angle, nz, n)
