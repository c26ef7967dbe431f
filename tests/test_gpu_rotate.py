"""GPU parity of projection rotation (tcb_rotate_proj) with the oracle's
restatement of scipy.ndimage's geometric transform (bit for bit against
scipy's rotate; the reference calls cupyx's rotate, a separate NVRTC-compiled
implementation that may fuse multiply-adds and is not installed here, so
agreement with the reference's own call is bounded by the 1e-5
reconstruction parity below, not shown bit for bit), and of
reconstructions with rotate_proj_angle set: the step driver (whole
projections) and GPURec.recon_all (each sinogram chunk, as the reference's
recon_all runs proc_proj) against the oracle's pre-processing fed to the
reference's CUDA filter and fourierrec."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("angle,shape", [(0.7, (5, 33, 70)), (-2.25, (3, 64, 257)),
                                         (15.0, (2, 17, 40)), (181.3, (4, 8, 9)),
                                         (1.0, (1, 2048, 2048))])
def test_rotate_kernel_matches_oracle(cuda, order, angle, shape):
    from oracle import np_tomo
    from tomocupy_b200.processing.proc_functions import rotate_proj
    rng = np.random.default_rng(3)
    data = rng.random(shape, dtype=np.float32) * 4 - 1
    got = rotate_proj(torch.as_tensor(data, device=cuda), angle, order).cpu().numpy()
    want = np_tomo.rotate_proj(data, angle, order)
    assert np.array_equal(got, want), np.abs(got - want).max()


def test_rotate_kernel_strided_frames(cuda):
    """Frames inside a taller buffer (frame stride > nz * n) and out != in."""
    from oracle import np_tomo
    from tomocupy_b200.processing.proc_functions import rotate_proj
    rng = np.random.default_rng(4)
    big = torch.as_tensor(rng.random((6, 12, 50), dtype=np.float32), device=cuda)
    view = big[:, :7]                                      # frame stride 12 * 50
    out = torch.full((6, 9, 50), 5.0, device=cuda)[:, :7]  # frame stride 9 * 50
    rotate_proj(view, -4.0, 1, out=out)
    want = np_tomo.rotate_proj(view.cpu().numpy(), -4.0, 1)
    assert np.array_equal(out.cpu().numpy(), want)


def test_rotate_rejects_bad_input(cuda):
    from tomocupy_b200.processing.proc_functions import rotate_proj
    x = torch.zeros((2, 8, 8), device=cuda)
    with pytest.raises(NotImplementedError):
        rotate_proj(x, 1.0, 3)
    with pytest.raises(Exception):
        rotate_proj(x, 1.0, 1, out=x)


def _ref_rec(ref, cuda, rows, theta, center, n):
    """The reference's filter + fourierrec of -log rows [nz, nproj, n]."""
    from oracle import np_tomo
    nz, nproj = rows.shape[:2]
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    filt = ref.RefFilter(ne, nproj, nz)
    rec = ref.RefFourierRec(n, nproj, nz, torch.as_tensor(theta, device=cuda))
    d = torch.as_tensor(np.ascontiguousarray(rows), device=cuda)
    d = ref.ref_fbp_filter_center(filt, d, wf, t, center, torch.zeros(nz, device=cuda), n, ne)
    out = torch.zeros((nz, n, n), device=cuda)
    rec.backprojection(out, d)
    return out.cpu()


def test_step_driver_rotation_matches_reference_chain(cuda, ref):
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec_steps import GPURecSteps
    nproj, nz, n = 120, 4, 128
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=21)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=4,
                      rotate_proj_angle=1.5)
    w = ArrayWriter(device="cuda")
    GPURecSteps(ArrayReader(data, dark, flat, theta=theta), w).recon_steps_all()
    pre = np_tomo.darkflat(data.numpy(), dark.numpy(), flat.numpy())
    pre = np_tomo.minus_log(np_tomo.rotate_proj(pre, 1.5, 1))         # [nproj, nz, n]
    theirs = _ref_rec(ref, cuda, pre.transpose(1, 0, 2), np.asarray(theta), params.center, n)
    assert rel_l2(w.rec.cpu(), theirs) < 1e-5


def test_recon_all_rotation_per_chunk_matches_reference_chain(cuda, ref):
    """Chunks of 4 rows, the last one partial (2 rows): each chunk rotated at
    the chunk height of 4 (zero rows below a partial chunk), then -log."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    nproj, nz, n, ncz, angle = 120, 6, 128, 4, -2.0
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=22)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=ncz,
                      rotate_proj_angle=angle)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_all()
    ours = w.rec.cpu()
    dfc = np_tomo.darkflat(data.numpy(), dark.numpy(), flat.numpy())
    for z0 in range(0, nz, ncz):
        lz = min(ncz, nz - z0)
        chunk = np.zeros((nproj, ncz, n), dtype=np.float32)
        chunk[:, :lz] = dfc[:, z0:z0 + lz]
        pre = np_tomo.minus_log(np_tomo.rotate_proj(chunk, angle, 1))
        pre[:, lz:] = 0
        theirs = _ref_rec(ref, cuda, pre.transpose(1, 0, 2), np.asarray(theta),
                          params.center, n)
        err = rel_l2(ours[z0:z0 + lz], theirs[:lz])
        assert err < 1e-5, (z0, err)
