"""GPU parity of the double-FOV padding (tcb_pad360_rows) against fixtures
made by the reference's own pad360, and of a double-FOV reconstruction
through GPURec against the reference's CUDA build fed with the restated
pre-processing and padding."""
import ctypes as C
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import PAD360_CASES
    return PAD360_CASES


@pytest.mark.parametrize("i", range(3))
def test_pad360_rows_match_reference_fixture(cuda, i):
    from tomocupy_b200 import _lib
    nproj, nz, ni, centeri, seed = _cases()[i]
    center = ni - centeri if centeri < ni // 2 else centeri
    g = np.load(ROOT / "tests" / "golden" / "pad360.npz")
    w = max(1, int(2 * (ni - center)))
    v = np.empty(w, dtype=np.float64)
    _lib.call("tcb_pad360_weights", v.ctypes.data_as(C.c_void_p), w)
    vd = torch.as_tensor(v, device=cuda)
    stride = 2 * ni + 3                       # rows wider than 2 ni: untouched tail
    rows = torch.full((nproj * nz, stride), 7.0, device=cuda)
    rows[:, :ni] = torch.as_tensor(g[f"in_{i}"], device=cuda).reshape(-1, ni)
    _lib.call("tcb_pad360_rows", rows.data_ptr(), nproj * nz, ni, stride,
              int(centeri < ni // 2), vd.data_ptr(), w, 0)
    torch.cuda.synchronize()
    got = rows.cpu().numpy()
    want = g[f"out_{i}"]
    out = got[:, :2 * ni].reshape(nproj, nz, 2 * ni)
    # bit for bit outside the transition; inside it the float64 weight may
    # differ from NumPy's in the last bit, so the float32 product by <= 1 ulp
    assert np.array_equal(out[:, :, :ni - w], want[:, :, :ni - w])
    assert np.array_equal(out[:, :, ni:], want[:, :, ni:])
    ulp = np.spacing(np.abs(want[:, :, ni - w:ni]))
    assert (np.abs(out[:, :, ni - w:ni] - want[:, :, ni - w:ni]) <= ulp).all()
    assert (got[:, 2 * ni:] == 7.0).all()


@pytest.mark.parametrize("axis", [118.0, 9.5])
def test_double_fov_reconstruction_matches_reference_chain(cuda, ref, axis):
    """360-degree scan, rotation axis near the right (no flip) or left (flip)
    edge: GPURec at n = 2 ni against dark/flat -> -log -> pad360 (restated)
    -> the reference's filter and fourierrec at the same centre."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    nproj, nz, ni = 180, 4, 128
    theta = np.linspace(0, 2 * np.pi, nproj, endpoint=False).astype(np.float32)
    data, dark, flat, _, _ = synthetic.make_dataset(nproj, nz, ni, seed=6, theta=theta)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=4,
                      file_type="double_fov", rotation_axis=axis)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_all()
    ours = w.rec.cpu()
    n, center = params.n, params.center
    assert n == 2 * ni
    pre = np_tomo.minus_log(np_tomo.darkflat(data.numpy(), dark.numpy(), flat.numpy()))
    pad = np_tomo.pad360(pre, params.centeri, ni, center)          # [nproj, nz, 2 ni]
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    filt = ref.RefFilter(ne, nproj, nz)
    rec = ref.RefFourierRec(n, nproj, nz, torch.as_tensor(theta, device=cuda))
    d = torch.as_tensor(np.ascontiguousarray(pad.transpose(1, 0, 2)), device=cuda)
    d = ref.ref_fbp_filter_center(filt, d, wf, t, center, torch.zeros(nz, device=cuda), n, ne)
    theirs = torch.zeros((nz, n, n), device=cuda)
    rec.backprojection(theirs, d)
    err = rel_l2(ours, theirs.cpu())
    assert err < 1e-5, err


def test_double_fov_try_sweep_matches_reference_chain(cuda, ref):
    """Try-centre sweep of a double-FOV scan (axis on the left: the shifts are
    inverted as Reader.init_sizes_try does) against dark/flat -> -log ->
    pad360 (restated) -> the reference's filter at each shift and its
    fourierrec."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    nproj, nz, ni = 180, 4, 128
    theta = np.linspace(0, 2 * np.pi, nproj, endpoint=False).astype(np.float32)
    data, dark, flat, _, _ = synthetic.make_dataset(nproj, nz, ni, seed=8, theta=theta)
    global_vars.reset(reconstruction_algorithm="fourierrec", reconstruction_type="try",
                      nsino_per_chunk=4, nsino="0.5", center_search_width=2.0,
                      center_search_step=1.0, file_type="double_fov", rotation_axis=9.5)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_try()
    zs, n, center = int(params.id_slices[0]), params.n, params.center
    shifts = np.asarray(params.shift_array, dtype=np.float32)
    assert n == 2 * ni and len(w.tries) == len(shifts)
    pre = np_tomo.minus_log(np_tomo.darkflat(data[:, zs:zs + 1].numpy(),
                                             dark[:, zs:zs + 1].numpy(),
                                             flat[:, zs:zs + 1].numpy()))
    pad = np_tomo.pad360(pre, params.centeri, ni, center)        # [nproj, 1, 2 ni]
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    filt = ref.RefFilter(ne, nproj, 4)
    rec = ref.RefFourierRec(n, nproj, 4, torch.as_tensor(theta, device=cuda))
    rows = torch.as_tensor(np.ascontiguousarray(pad.transpose(1, 0, 2)), device=cuda)
    for k in range(0, len(shifts), 4):
        cnt = min(4, len(shifts) - k)
        sht = torch.zeros(4, device=cuda)
        sht[:cnt] = torch.as_tensor(shifts[k:k + cnt], device=cuda)
        d = rows.expand(4, -1, -1).contiguous()
        d = ref.ref_fbp_filter_center(filt, d, wf, t, center, sht, n, ne)
        theirs = torch.zeros((4, n, n), device=cuda)
        rec.backprojection(theirs, d)
        for kk in range(cnt):
            ours = w.tries[(zs, float(params.save_centers[k + kk]))].cpu()
            err = rel_l2(ours, theirs[kk].cpu())
            assert err < 1e-4, (k + kk, err)


@pytest.mark.parametrize("axis,stripe,dz", [(118.0, "none", 0), (9.5, "none", 0),
                                            (118.0, "fw", 0), (9.5, "ti", 0),
                                            (118.0, "none", 3), (9.5, "ti", 5)])
def test_step_driver_double_fov_matches_recon_all(cuda, axis, stripe, dz):
    """GPURecSteps pads whole pre-processed projections (pad360 after -log) and
    backprojects; GPURec.recon_all pads each chunk's filter rows.  Ring
    removal runs on the ni-wide sinograms before the padding in both
    (proc_sino before proc_proj, proc_functions.py:140-195).  Same operations
    in the same order: the volumes agree to float32 rounding."""
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    from tomocupy_b200.rec_steps import GPURecSteps
    nproj, nz, ni = 120, 8, 96
    theta = np.linspace(0, 2 * np.pi, nproj, endpoint=False).astype(np.float32)
    data, dark, flat, _, _ = synthetic.make_dataset(nproj, nz, ni, seed=9, theta=theta)
    if dz:  # outlier removal runs on the ni-wide raw frames before the padding
        d32 = data.to(torch.int32)
        d32.view(-1)[torch.as_tensor(np.random.default_rng(2).integers(0, data.numel(), 200))] = 60000
        data = d32.to(torch.uint16)
    opts = dict(reconstruction_algorithm="fourierrec", nsino_per_chunk=4,
                file_type="double_fov", rotation_axis=axis, remove_stripe_method=stripe,
                fw_level=4, dezinger=dz)
    global_vars.reset(**opts)
    w1 = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w1).recon_all()
    a = w1.rec.cpu()
    global_vars.reset(**opts)
    w2 = ArrayWriter(device="cuda")
    GPURecSteps(ArrayReader(data, dark, flat, theta=theta), w2).recon_steps_all()
    b = w2.rec.cpu()
    assert a.shape == b.shape == (nz, 2 * ni, 2 * ni)
    assert rel_l2(b, a) < (1e-6 if stripe == "none" else 1e-5)
