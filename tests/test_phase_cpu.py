"""Phase retrieval on the CPU: the NumPy restatement (oracle.np_tomo) against
fixtures made by the reference's own paganin_filter / farago_filter
(src/tomocupy/processing/retrieve_phase.py, executed with NumPy for CuPy by
tests/golden/make_golden.py), the library's host-side padding rule against
the same fixtures, and the identity the native operator is built on."""
import ctypes as C
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_l2


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import PHASE_CASES
    return PHASE_CASES


def _golden():
    return np.load(ROOT / "tests" / "golden" / "phase_retrieval.npz")


@pytest.mark.parametrize("i", range(6))
def test_oracle_matches_reference_fixture(i):
    from oracle import np_tomo
    meth, nproj, dy, dz, ps, dist, en, alpha, db, W, seed = _cases()[i]
    g = _golden()
    got = np_tomo.retrieve_phase(g[f"in_{i}"], meth, ps, dist, en, alpha, db, W)
    assert got.dtype == np.float32 and got.shape == (nproj, dy, dz)
    assert rel_l2(got, g[f"out_{i}"]) < 1e-6


@pytest.mark.parametrize("i", range(6))
def test_library_pads_match_reference(i):
    """tcb_phase_pads (host arithmetic only) against _calc_pad's choice."""
    from tomocupy_b200 import _lib
    meth, nproj, dy, dz, ps, dist, en, alpha, db, W, seed = _cases()[i]
    py, pz = C.c_size_t(), C.c_size_t()
    _lib.call("tcb_phase_pads", dy, dz, ps, dist, en, 1, C.byref(py), C.byref(pz))
    assert [py.value, pz.value] == list(_golden()[f"pads_{i}"])


def test_pads_sweep_matches_oracle():
    from oracle import np_tomo
    from tomocupy_b200.processing.retrieve_phase import pads
    rng = np.random.default_rng(0)
    for _ in range(200):
        dy, dz = (int(v) for v in rng.integers(1, 5000, 2))
        ps = float(rng.uniform(0.3e-4, 5e-4))
        dist, en = float(rng.uniform(0, 100)), float(rng.uniform(5, 80))
        assert pads(dy, dz, ps, dist, en) == np_tomo.pr_pads(dy, dz, ps, dist, en)
    assert pads(100, 60, 1e-4, 5.0, 20.0, pad=False) == (0, 0)


def test_bad_arguments_are_rejected():
    from tomocupy_b200 import _lib
    from tomocupy_b200.processing.retrieve_phase import pads
    with pytest.raises(_lib.TcbError):
        pads(64, 64, 0.0, 5.0, 20.0)       # the reference divides by pixel_size**2
    with pytest.raises(_lib.TcbError):
        pads(0, 64, 1e-4, 5.0, 20.0)


@pytest.mark.parametrize("method", ["paganin", "Gpaganin", "farago"])
def test_even_filter_identity(method):
    """real(ifft2(fft2(p) * F)) == ifft2(fft2(p) * Fe), Fe(k) = (F(k) + F(-k)) / 2,
    for the reference's (not centro-symmetric) shifted filters: the native
    operator's R2C / C2R form (float64 here, to isolate the identity)."""
    from oracle import np_tomo
    rng = np.random.default_rng(1)
    ny, nz = 40, 56
    p = rng.random((ny, nz))
    f = np_tomo.pr_filter(method, ny, nz, 1e-4, 0.5, 25.0, 1e-3, 1000.0, 2e-4).astype(np.float64)
    f = f / f.max()
    fe = 0.5 * (f + np.roll(f[::-1, ::-1], (1, 1), axis=(0, 1)))
    assert np.abs(f - fe).max() > 1e-3   # the filter itself is not even
    a = np.real(np.fft.ifft2(np.fft.fft2(p) * f))
    b = np.fft.irfft2(np.fft.rfft2(p) * fe[:, :nz // 2 + 1], s=(ny, nz))
    assert np.abs(a - b).max() < 1e-12
