"""GPU parity of the log-polar backprojector against the reference CUDA build.

The reference operator runs on the grids produced by the reference's own
Python (tests/golden/lprec_grids.npz); ours builds its grids itself.  Both
use hardware-filtered texture fetches, so the remaining differences come
from the float32 order of the prefilter/FFT arithmetic: rel-L2 <= 1e-5.
"""
import numpy as np
import pytest
import torch

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu

GOLD = ROOT / "tests" / "golden" / "lprec_grids.npz"


def _golden(n, nproj):
    g = np.load(GOLD)
    keys = ("fZ", "lp2p1", "lp2p2", "lp2p1w", "lp2p2w", "C2lp1", "C2lp2", "cids", "lpids",
            "wids")
    return {k: g[f"{k}_{n}_{nproj}"] for k in keys}


@pytest.mark.parametrize("n,nproj,nz", [(128, 90, 4), (200, 128, 2)])
def test_lprec_vs_reference(cuda, ref, n, nproj, nz):
    from tomocupy_b200.reconstruction.lprec import LpRec
    theta = (np.arange(nproj) * np.pi / nproj).astype(np.float32)
    rng = np.random.default_rng(n)
    data = torch.as_tensor(rng.standard_normal((nz, nproj, n)).astype(np.float32), device=cuda)
    fa = torch.empty((nz, n, n), device=cuda)
    LpRec(n, nproj, nz, theta, "float32").backprojection(fa, data.clone())
    fb = torch.empty((nz, n, n), device=cuda)
    ref.RefLpRec(n, nproj, nz, _golden(n, nproj)).backprojection(fb, data.clone())
    torch.cuda.synchronize()
    err = rel_l2(fa.cpu(), fb.cpu())
    assert err < 1e-5, err


def test_lprec_fp16_storage(cuda):
    from tomocupy_b200.reconstruction.lprec import LpRec
    n, nproj, nz = 128, 90, 2
    theta = (np.arange(nproj) * np.pi / nproj).astype(np.float32)
    rng = np.random.default_rng(3)
    data = torch.as_tensor(rng.standard_normal((nz, nproj, n)).astype(np.float32), device=cuda)
    f32 = torch.empty((nz, n, n), device=cuda)
    LpRec(n, nproj, nz, theta, "float32").backprojection(f32, data.clone())
    f16 = torch.empty((nz, n, n), dtype=torch.float16, device=cuda)
    LpRec(n, nproj, nz, theta, "float16").backprojection(f16, data.clone().half())
    torch.cuda.synchronize()
    assert rel_l2(f16.float().cpu(), f32.cpu()) < 5e-3


def test_lprec_rejects_uneven_angles():
    from tomocupy_b200.reconstruction import lprec_grids
    with pytest.raises(ValueError):
        lprec_grids.check_angles(np.linspace(0, np.pi, 90), 90)  # includes the endpoint


@pytest.mark.parametrize("n,nproj,nz", [(256, 256, 4), (512, 400, 3)])
def test_lprec_own_fft_vs_reference_and_cufft(cuda, ref, monkeypatch, n, nproj, nz):
    """Power-of-two log-polar grids of at least 256 run the FFT convolution
    on the library's own FFT (two slices packed as one complex image; an odd
    slice count leaves the last pair half empty).  Against the reference
    build (fed the same grids, which are bit-exact with the reference's own)
    within the lprec tolerance, and against the cuFFT R2C/C2R chain
    (TCB_LPREC_FFT set) to float rounding."""
    from tomocupy_b200.reconstruction import lprec_grids as L
    from tomocupy_b200.reconstruction.lprec import LpRec
    theta = (np.arange(nproj) * np.pi / nproj).astype(np.float32)
    rng = np.random.default_rng(n)
    data = torch.as_tensor(rng.standard_normal((nz, nproj, n)).astype(np.float32), device=cuda)
    own = torch.empty((nz, n, n), device=cuda)
    LpRec(n, nproj, nz, theta, "float32").backprojection(own, data.clone())
    monkeypatch.setenv("TCB_LPREC_FFT", "cufft")
    lib = torch.empty((nz, n, n), device=cuda)
    LpRec(n, nproj, nz, theta, "float32").backprojection(lib, data.clone())
    ntheta, nrho = L.lp_sizes(n, nproj)
    grids = vars(L.create_adj(L.create_gl(n, nproj, ntheta, nrho)))
    theirs = torch.empty((nz, n, n), device=cuda)
    ref.RefLpRec(n, nproj, nz, grids).backprojection(theirs, data.clone())
    torch.cuda.synchronize()
    e_lib = rel_l2(own.cpu(), lib.cpu())
    e_ref = rel_l2(own.cpu(), theirs.cpu())
    print(f"lprec own FFT {n}x{nproj}: vs cuFFT chain {e_lib:.2e}, vs reference {e_ref:.2e}")
    assert e_lib < 1e-6, e_lib
    assert e_ref < 1e-5, e_ref
