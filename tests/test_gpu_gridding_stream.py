"""Tensor-core gridding with streamed weights (TCB_GRID_TENSOR_FP32 and
TCB_GRID_TENSOR_STREAM) against the reference's CUDA build and the fp32
register gridding.

The fp32 drop-in form multiplies split-fp16 operands (W_hi V_hi + W_lo V_hi +
W_hi V_lo, fp32 accumulation in TMEM): within the fourierrec tolerance of
the reference (1e-5, the reference sums with unordered atomics); the mixed
form (fp16 weights and values) within the 1e-3 mixed-precision budget of
the fp32 path."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _theta(nproj, kind="uniform", seed=0):
    if kind == "uniform":
        return (np.arange(nproj) * np.pi / nproj).astype(np.float32)
    rng = np.random.default_rng(seed)
    return np.sort(rng.uniform(0, np.pi, nproj)).astype(np.float32)


def _run(cuda, n, nproj, nz, theta, g, mode):
    from tomocupy_b200 import cfunc_fourierrec
    op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
    op.set_gridding(mode)
    f = torch.full((nz, n, n, 2), float("nan"), device=cuda)
    op.backprojection(f, g.clone(), None)
    torch.cuda.synchronize()
    assert not op.timed_out()
    op.free()
    return f.cpu()


CASES = [(128, 90, 2, "uniform"), (200, 120, 3, "random"), (512, 360, 40, "uniform"),
         (256, 401, 70, "random"), (2048, 150, 2, "uniform"), (2048, 1500, 4, "uniform")]


@pytest.mark.parametrize("n,nproj,nz,kind", CASES)
def test_tensor_fp32_gridding_vs_reference(cuda, ref, n, nproj, nz, kind):
    """Partial tiles (n = 200), one and two pair groups (N = 64 and 128, more
    than 64 pairs), the production geometry."""
    from tomocupy_b200 import _lib
    theta = torch.as_tensor(_theta(nproj, kind, seed=n), device=cuda)
    g = torch.randn((nz, nproj, n, 2), device=cuda)
    ours = _run(cuda, n, nproj, nz, theta, g, _lib.GRID_TENSOR_FP32)
    assert torch.isfinite(ours).all()
    fp32 = _run(cuda, n, nproj, nz, theta, g, _lib.GRID_FP32)
    if nz * (2 * n + 8) ** 2 < 2 ** 31:
        f_ref = torch.empty((nz, n, n, 2), device=cuda)
        L = ref.lib("fourierrec")
        h = L.ref_create(nproj, nz, n, theta.data_ptr())
        L.ref_backprojection(h, f_ref.data_ptr(), g.clone().data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        L.ref_destroy(h)
        err = rel_l2(ours, f_ref.cpu())
        print(f"tensor fp32 gridding n={n} nproj={nproj} nz={nz}: vs reference {err:.2e}, "
              f"vs fp32 gridding {rel_l2(ours, fp32):.2e}")
        assert err < 1e-5, err
    assert rel_l2(ours, fp32) < 1e-5


@pytest.mark.parametrize("n,nproj,nz", [(128, 90, 2), (512, 360, 40), (2048, 150, 2)])
def test_tensor_stream_mixed_vs_fp32(cuda, n, nproj, nz):
    from tomocupy_b200 import _lib
    theta = torch.as_tensor(_theta(nproj, "random"), device=cuda)
    g = torch.randn((nz, nproj, n, 2), device=cuda) * 100.0
    mixed = _run(cuda, n, nproj, nz, theta, g, _lib.GRID_TENSOR_STREAM)
    fp32 = _run(cuda, n, nproj, nz, theta, g, _lib.GRID_FP32)
    err = rel_l2(mixed, fp32)
    print(f"streamed mixed gridding n={n}: vs fp32 {err:.2e}")
    assert torch.isfinite(mixed).all() and err < 1e-3, err


def test_tensor_fp32_gridding_deterministic(cuda):
    from tomocupy_b200 import _lib, cfunc_fourierrec
    n, nproj, nz = 256, 180, 6
    theta = torch.as_tensor(_theta(nproj), device=cuda)
    g = torch.randn((nz, nproj, n, 2), device=cuda)
    op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
    op.set_gridding(_lib.GRID_TENSOR_FP32)
    outs = []
    for _ in range(2):
        f = torch.empty((nz, n, n, 2), device=cuda)
        op.backprojection(f, g.clone(), None)
        outs.append(f.cpu())
    assert not op.timed_out()
    op.free()
    assert torch.equal(outs[0], outs[1])
