"""GPU check of the Fourier-wavelet ring removal against fixtures produced by
the reference's own remove_stripe_fw (executed with NumPy for CuPy; the
filter banks come from tomocupy_b200.processing.wavelets because PyWavelets
is not available, see tests/golden/make_golden.py).  The wavelet stages use
the reference's float32 operation order; the band FFTs differ (cuFFT float32
here, NumPy float64 in the fixture), hence rel-L2 <= 1e-5."""
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu


def _cases():
    import sys
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import FW_CASES
    return FW_CASES


@pytest.mark.parametrize("i", range(4))
def test_fw_matches_reference_fixture(cuda, i):
    from tomocupy_b200.processing.remove_stripe import remove_stripe_fw
    g = np.load(ROOT / "tests" / "golden" / "fw_stripe.npz")
    nproj, nz, n, level, sigma, wname, seed = _cases()[i]
    data = torch.as_tensor(g[f"in_{i}"], device=cuda)
    out = remove_stripe_fw(data, sigma, wname, level)
    torch.cuda.synchronize()
    want = g[f"out_{i}"]
    assert out.shape == want.shape
    err = rel_l2(out.cpu().numpy(), want)
    assert err < 1e-5, (i, err)


@pytest.fixture
def cufft_damping(monkeypatch):
    """fw operators built with the band damping on cuFFT (TCB_FW_DAMP)."""
    from tomocupy_b200.processing import remove_stripe
    monkeypatch.setenv("TCB_FW_DAMP", "cufft")
    remove_stripe._operator.cache_clear()
    yield
    remove_stripe._operator.cache_clear()


@pytest.mark.parametrize("i", range(5))
def test_fw_filter_banks_reproduce_regression_fixture(cuda, cufft_damping, i):
    """Bit-for-bit against outputs recorded with the one-output-per-thread
    filter-bank kernels and the cuFFT band damping
    (tests/golden/make_fw_b200.py): the register-blocked kernels keep every
    output's multiply-then-add tap order."""
    import sys
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_fw_b200 import CASES
    from tomocupy_b200.processing.remove_stripe import remove_stripe_fw
    g = np.load(ROOT / "tests" / "golden" / "fw_stripe_b200.npz")
    nproj, nz, n, level, sigma, wname, seed = CASES[i]
    out = remove_stripe_fw(torch.as_tensor(g[f"in_{i}"], device=cuda), sigma, wname, level)
    torch.cuda.synchronize()
    want = g[f"out_{i}"]
    got = out.cpu().numpy()
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), \
        (i, float(np.abs(got - want).max()))


@pytest.mark.parametrize("nproj,nz,n,level,sigma", [
    (1500, 2, 2048, 7, 1.0),     # production sizes: bands of 859 (odd) ... rows
    (720, 3, 1024, 5, 2.0),
    (181, 2, 256, 3, 3.0),       # wide Gaussian: 32 modes, short bands on cuFFT
])
def test_fw_mode_damping_matches_cufft(cuda, monkeypatch, nproj, nz, n, level, sigma):
    """The band damping by projection onto the Gaussian's few Fourier modes
    equals the rfft -> multiply -> irfft damping (cuFFT) to float rounding."""
    from tomocupy_b200.processing import remove_stripe
    from tomocupy_b200 import synthetic
    data, dark, flat, _, _ = synthetic.make_dataset(nproj, nz, n, seed=4, stripes=12)
    x = (data.to(torch.float32) / 1000.0).to(cuda)
    remove_stripe._operator.cache_clear()
    modes = remove_stripe.remove_stripe_fw(x, sigma, "sym16", level)
    monkeypatch.setenv("TCB_FW_DAMP", "cufft")
    remove_stripe._operator.cache_clear()
    fft = remove_stripe.remove_stripe_fw(x, sigma, "sym16", level)
    remove_stripe._operator.cache_clear()
    err = rel_l2(modes.cpu(), fft.cpu())
    print(f"fw mode damping vs cuFFT {nproj}x{n} level {level} sigma {sigma}: {err:.2e}")
    assert err < 1e-6, err


def test_fw_removes_stripes(cuda):
    """Constant-along-angle column offsets are strongly attenuated."""
    from tomocupy_b200.processing.remove_stripe import remove_stripe_fw
    rng = np.random.default_rng(0)
    nproj, nz, n = 180, 2, 256
    smooth = np.exp(-np.linspace(-2, 2, n) ** 2)[None, None, :] * np.ones((nproj, nz, 1))
    stripes = np.zeros(n)
    stripes[rng.choice(n, 12, replace=False)] = 0.05
    data = torch.as_tensor((smooth + stripes[None, None, :]).astype(np.float32), device=cuda)
    out = remove_stripe_fw(data, 1.0, "sym16", 5).cpu().numpy()
    before = np.abs(np.diff(data.cpu().numpy().mean(0), axis=-1)).max()
    after = np.abs(np.diff(out.mean(0), axis=-1)).max()
    assert after < 0.5 * before


def _ti_cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import TI_CASES
    return TI_CASES


@pytest.mark.parametrize("i", range(4))
def test_ti_matches_reference_fixture(cuda, i):
    """Titarenko ring removal against the reference's own remove_stripe_ti
    (NumPy for CuPy): float32 column means (double accumulation here), the
    gamma convolution in float64, the add rounded once to float32."""
    from tomocupy_b200.processing.remove_stripe import remove_stripe_ti
    g = np.load(ROOT / "tests" / "golden" / "ti_stripe.npz")
    nproj, nz, n, beta, mask, seed = _ti_cases()[i]
    data = torch.as_tensor(g[f"in_{i}"], device=cuda)
    out = remove_stripe_ti(data, beta, mask)
    torch.cuda.synchronize()
    assert out.data_ptr() == data.data_ptr()
    want = g[f"out_{i}"]
    assert rel_l2(out.cpu().numpy(), want) < 1e-6
    assert float(np.abs(out.cpu().numpy() - want).max()) < 1e-6


def test_ti_float_mask_and_larger_size(cuda):
    """A float mask size (which the reference's slicing rejects) selects the
    same centred columns as the oracle's integer-cast slice; 2048 columns."""
    from oracle import np_tomo
    from tomocupy_b200.processing.remove_stripe import remove_stripe_ti
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import ti_input
    x = ti_input(300, 3, 2048, seed=11)
    want = np_tomo.remove_stripe_ti(x, 0.022, 0.5)
    got = remove_stripe_ti(torch.as_tensor(x, device=cuda), 0.022, 0.5).cpu().numpy()
    assert rel_l2(got, want) < 1e-6
    assert np.array_equal(got[:, :, :512], x[:, :, :512])   # outside the mask: untouched


def test_ti_rejects_odd_width(cuda):
    from tomocupy_b200 import _lib
    from tomocupy_b200.processing.remove_stripe import remove_stripe_ti
    with pytest.raises(_lib.TcbError):
        remove_stripe_ti(torch.ones((4, 2, 101), device=cuda), 0.022, 1)
