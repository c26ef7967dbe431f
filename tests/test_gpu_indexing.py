"""Bit-exact indexing against the reference's own CUDA build.

The reference places every polar sample with its own kernels: takexy for
fourierrec (src/include/kernels_fourierrec.cuh:23-36) and take_x for the
laminography usfft2d (src/include/kernels_usfft2d.cu:5-18).  The shims in
oracle/ref_shims launch exactly those kernels; the library exports the
positions its gridding kernels use.  They must agree bit for bit, as must
the footprint origins floor(2n x) that follow from them.

linerec computes its detector indices (ur, vr), weights and sums inside
one kernel (src/include/kernels_linerec.cuh:3-46); the library writes the
same roundings out explicitly, so outputs are compared bit for bit.
"""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _theta(nproj, kind, seed=0):
    if kind == "uniform":
        return (np.arange(nproj) * np.pi / nproj).astype(np.float32)
    rng = np.random.default_rng(seed)
    return np.sort(rng.uniform(0, np.pi, nproj)).astype(np.float32)


@pytest.mark.parametrize("n", [512, 2048])
@pytest.mark.parametrize("kind", ["uniform", "random"])
def test_fourierrec_sample_positions_bit_exact(cuda, ref, n, kind):
    from tomocupy_b200 import cfunc_fourierrec
    nproj = 1500
    theta = torch.as_tensor(_theta(nproj, kind, seed=n), device=cuda)
    op = cfunc_fourierrec.cfunc_fourierrec(nproj, 1, n, theta)
    x, y, fx, fy = op.sample_positions()
    xr = torch.empty((nproj, n), dtype=torch.float32, device=cuda)
    yr = torch.empty_like(xr)
    ref.lib("fourierrec").ref_takexy(xr.data_ptr(), yr.data_ptr(), theta.data_ptr(), n, nproj,
                                     torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    op.free()
    assert torch.equal(x.cpu(), xr.cpu())
    assert torch.equal(y.cpu(), yr.cpu())
    # footprint origins: (int)floorf(2 * n * x) (kernels_fourierrec.cuh:84-85)
    two_n = np.float32(2 * n)
    want_fx = np.floor(two_n * xr.cpu().numpy()).astype(np.int32)
    want_fy = np.floor(two_n * yr.cpu().numpy()).astype(np.int32)
    assert np.array_equal(fx.cpu().numpy(), want_fx)
    assert np.array_equal(fy.cpu().numpy(), want_fy)


@pytest.mark.parametrize("lamino_deg,k", [(30.0, 3), (-20.0, 0), (0.0, 1), (61.5, 7)])
def test_usfft2d_sample_positions_bit_exact(cuda, ref, lamino_deg, k):
    from tomocupy_b200 import cfunc_usfft2d
    ntheta, detw, deth, deth0, n = 1200, 1024, 16, 1024, 1024
    theta = torch.as_tensor(np.linspace(0, 2 * np.pi, ntheta, endpoint=False,
                                        dtype=np.float32), device=cuda)
    phi = float(np.float32(math.pi / 2 + lamino_deg / 180 * math.pi))
    # cfunc_usfft2d(n0, n1, n2, ntheta, detw, deth) in the reference's Python order
    op = cfunc_usfft2d.cfunc_usfft2d(deth, n, n, ntheta, detw, deth)
    x = torch.empty((ntheta, deth, detw), dtype=torch.float32, device=cuda)
    y = torch.empty_like(x)
    op.sample_positions(x, y, theta, phi, k, deth0, None)
    xr = torch.empty_like(x)
    yr = torch.empty_like(x)
    ref.lib("usfft2d").ref_take_x(xr.data_ptr(), yr.data_ptr(), theta.data_ptr(), phi, k, deth0,
                                  detw, deth, ntheta, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    op.free()
    assert torch.equal(x.cpu(), xr.cpu())
    assert torch.equal(y.cpu(), yr.cpu())


@pytest.mark.parametrize("lamino_deg", [0.0, 20.0, -35.0])
@pytest.mark.parametrize("nproj", [1, 60])
def test_linerec_bit_identical_to_reference(cuda, ref, lamino_deg, nproj):
    """One angle (every special angle on its own) and 60 angles: the detector
    indices, weights and per-voxel sums equal the reference build's bit for
    bit (the kernels write out the reference's roundings)."""
    from tomocupy_b200.reconstruction.linerec import LineRec
    n, nz, ncz, sz = 256, 24, 4, 7   # slice offsets z = tz + sz - nz/2 in [-5, -2]
    g = torch.Generator(device="cpu").manual_seed(3)
    if nproj == 1:
        cases = [np.float32([t]) for t in (0.0, np.pi / 4, np.pi / 2, 3 * np.pi / 4,
                                           np.pi - 1e-3, 1e-6, 0.3)]
    else:
        cases = [_theta(nproj, "random", seed=7)]
    for th_np in cases:
        th = torch.as_tensor(th_np, device=cuda)
        data = (torch.rand((nz, nproj, n), generator=g) + 0.5).to(cuda)
        ours = LineRec(th, nproj, nproj, nz, ncz, n, "float32")
        theirs = ref.RefLineRec(th, nproj, nproj, nz, ncz, n)
        fa = torch.zeros((ncz, n, n), device=cuda)
        fb = torch.zeros((ncz, n, n), device=cuda)
        ours.backprojection(fa, data, None, th, lamino_angle=lamino_deg, sz=sz)
        theirs.backprojection(fb, data, None, th, lamino_angle=lamino_deg, sz=sz)
        torch.cuda.synchronize()
        assert torch.equal(fa.cpu(), fb.cpu()), (float(th_np[0]), int((fa != fb).sum()))
