"""GPU parity of the native phase retrieval (tcb_phase_*, through
tomocupy_b200.processing.retrieve_phase) against fixtures made by the
reference's own paganin_filter / farago_filter (NumPy for CuPy, complex64
transforms) and against the NumPy restatement on larger, production-like
geometries.  The native chain is R2C -> even part of the filter -> C2R in
float32 (cuFFT), the reference's a complex64 fft2 -> filter -> ifft2 -> real
part: equal in exact arithmetic, so the tolerance is float32 transform
rounding, rel-L2 <= 1e-5."""
import sys

import numpy as np
import pytest
import torch

from conftest import TorchCuFFT, ROOT, rel_l2

pytestmark = pytest.mark.gpu


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import PHASE_CASES
    return PHASE_CASES


def _run(data, meth, ps, dist, en, alpha, db, W, **kw):
    from tomocupy_b200.processing.retrieve_phase import PhaseFilter
    op = PhaseFilter(data.shape[1], data.shape[2], meth, ps, dist, en, alpha, db, W, **kw)
    out = op.apply(data)
    torch.cuda.synchronize()
    op.free()
    return out


@pytest.mark.parametrize("i", range(6))
def test_phase_matches_reference_fixture(cuda, i):
    g = np.load(ROOT / "tests" / "golden" / "phase_retrieval.npz")
    meth, nproj, dy, dz, ps, dist, en, alpha, db, W, seed = _cases()[i]
    data = torch.as_tensor(g[f"in_{i}"], device=cuda).contiguous()
    out = _run(data, meth, ps, dist, en, alpha, db, W)
    assert out.data_ptr() == data.data_ptr()          # in place, like data[m] = proj
    want = g[f"out_{i}"]
    err = rel_l2(out.cpu().numpy(), want)
    assert err < 1e-5, (i, meth, err)


@pytest.mark.parametrize("meth,shape,ps,dist,en", [
    ("paganin", (3, 300, 412), 0.65e-4, 5.0, 20.0),     # production optics, odd pads
    ("Gpaganin", (2, 256, 256), 0.65e-4, 5.0, 20.0),
    ("farago", (2, 200, 333), 1e-4, 0.5, 25.0),
])
def test_phase_matches_oracle_larger(cuda, meth, shape, ps, dist, en):
    from oracle import np_tomo
    _cases()
    from make_golden import phase_input
    x = phase_input(*shape, seed=7)
    want = np_tomo.retrieve_phase(x, meth, ps, dist, en, 1e-3, 1500.0, 1.3e-4)
    got = _run(torch.as_tensor(x, device=cuda), meth, ps, dist, en, 1e-3, 1500.0, 1.3e-4)
    err = rel_l2(got.cpu().numpy(), want)
    assert err < 1e-5, (meth, err)


def test_phase_batches_are_independent(cuda):
    """5 projections through batches of 2 (a partial last batch running the
    full-batch plan) equal one batch of 5, and a projection's result does not
    depend on its neighbours."""
    _cases()
    from make_golden import phase_input
    x = torch.as_tensor(phase_input(5, 48, 64, seed=9), device=cuda)
    args = ("paganin", 0.65e-4, 5.0, 20.0, 1e-3, 1500.0, 2e-4)
    a = _run(x.clone(), *args, batch=2)
    b = _run(x.clone(), *args, batch=5)
    c = _run(x[3:4].clone(), *args, batch=1)
    assert rel_l2(a.cpu(), b.cpu()) < 1e-6
    assert rel_l2(c[0].cpu(), b[3].cpu()) < 1e-6


def test_phase_rejects_bad_input(cuda):
    from tomocupy_b200.processing.retrieve_phase import PhaseFilter, paganin_filter
    op = PhaseFilter(16, 24, "paganin", 1e-4, 5.0, 20.0)
    with pytest.raises(ValueError):
        op.apply(torch.zeros((2, 16, 25), device=cuda))
    with pytest.raises(ValueError):
        op.apply(torch.zeros((2, 16, 24), device=cuda, dtype=torch.float64))
    op.free()
    with pytest.raises(ValueError):
        paganin_filter(torch.zeros((1, 8, 8), device=cuda), method="farago")


def test_step_driver_with_phase_retrieval(cuda):
    """GPURecSteps with Paganin phase retrieval (dark/flat -> phase -> -log ->
    filter -> fourierrec) against the same chain with the NumPy restatement's
    phase retrieval feeding the library's own reconstruction."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    from tomocupy_b200.rec_steps import GPURecSteps
    nproj, nz, n = 90, 16, 128
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=4)
    opts = dict(reconstruction_algorithm="fourierrec", nsino_per_chunk=8,
                retrieve_phase_method="paganin", pixel_size=0.65, propagation_distance=50.0,
                energy=20.0, retrieve_phase_alpha=1e-3)
    global_vars.reset(**opts)
    w = ArrayWriter(device="cuda")
    got = GPURecSteps(ArrayReader(data, dark, flat, theta=theta), w).recon_steps_all()
    got = w.rec.cpu().numpy() if got is None else got.cpu().numpy()
    # the same chain with the NumPy phase retrieval in the middle
    pre = np_tomo.darkflat(data.numpy(), dark.numpy(), flat.numpy())
    pre = np_tomo.retrieve_phase(pre, "paganin", 0.65e-4, 5.0, 20.0, 1e-3)
    pre = np_tomo.minus_log(pre)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=8)
    w2 = ArrayWriter(device="cuda")
    rec = GPURec(ArrayReader(data, dark, flat, theta=theta), w2)
    want = rec.recon_preprocessed(torch.as_tensor(pre, device=cuda)).cpu().numpy()
    err = rel_l2(got, want)
    assert np.isfinite(got).all() and err < 1e-4, err


def test_recon_all_phase_retrieval_per_chunk_matches_reference(cuda, ref):
    """GPURec.recon_all with Paganin phase retrieval applies it to each
    sinogram chunk's projections (rows of the chunk as the image height), as
    the reference's recon_all does (rec.py:170-173): against dark/flat ->
    restated paganin_filter per chunk -> -log -> the reference's CUDA filter
    and fourierrec."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    nproj, nz, n, ncz = 90, 16, 128, 8
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=12)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=ncz,
                      retrieve_phase_method="paganin", pixel_size=0.65,
                      propagation_distance=50.0, energy=20.0, retrieve_phase_alpha=1e-3)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_all()
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    filt = ref.RefFilter(ne, nproj, ncz)
    rec = ref.RefFourierRec(n, nproj, ncz, torch.as_tensor(theta, device=cuda))
    for z0 in range(0, nz, ncz):
        sl = slice(z0, z0 + ncz)
        pre = np_tomo.darkflat(data[:, sl].numpy(), dark[:, sl].numpy(), flat[:, sl].numpy())
        pre = np_tomo.minus_log(np_tomo.retrieve_phase(pre, "paganin", 0.65e-4, 5.0, 20.0, 1e-3))
        d = torch.as_tensor(np.ascontiguousarray(pre.transpose(1, 0, 2)), device=cuda)
        d = ref.ref_fbp_filter_center(filt, d, wf, t, n / 2, torch.zeros(ncz, device=cuda), n, ne)
        theirs = torch.zeros((ncz, n, n), device=cuda)
        rec.backprojection(theirs, d)
        err = rel_l2(w.rec[sl].cpu(), theirs.cpu())
        assert err < 1e-4, (z0, err)


def test_recon_all_ring_removal_then_phase_matches_reference(cuda, ref):
    """recon_all with Titarenko ring removal and Paganin phase retrieval: per
    chunk dark/flat -> ring removal -> phase retrieval -> -log (proc_sino then
    proc_proj), against the same order with the restated phase retrieval
    (the NumPy restatement of the ring removal reproduces the reference's
    remove_stripe_ti fixtures bit for bit, tests/test_stripe_ti_cpu.py)."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    nproj, nz, n, ncz = 90, 16, 128, 8
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=13, stripes=6)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=ncz,
                      remove_stripe_method="ti", ti_beta=0.022, ti_mask=1,
                      retrieve_phase_method="paganin", pixel_size=0.65,
                      propagation_distance=50.0, energy=20.0, retrieve_phase_alpha=1e-3)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_all()
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    filt = ref.RefFilter(ne, nproj, ncz)
    rec = ref.RefFourierRec(n, nproj, ncz, torch.as_tensor(theta, device=cuda))
    for z0 in range(0, nz, ncz):
        sl = slice(z0, z0 + ncz)
        pre = np_tomo.darkflat(data[:, sl].numpy(), dark[:, sl].numpy(), flat[:, sl].numpy())
        pre = np_tomo.remove_stripe_ti(pre, 0.022, 1, fft=TorchCuFFT)
        pre = np_tomo.minus_log(np_tomo.retrieve_phase(pre, "paganin", 0.65e-4, 5.0, 20.0, 1e-3))
        d = torch.as_tensor(np.ascontiguousarray(pre.transpose(1, 0, 2)), device=cuda)
        d = ref.ref_fbp_filter_center(filt, d, wf, t, n / 2, torch.zeros(ncz, device=cuda), n, ne)
        theirs = torch.zeros((ncz, n, n), device=cuda)
        rec.backprojection(theirs, d)
        err = rel_l2(w.rec[sl].cpu(), theirs.cpu())
        assert err < 1e-4, (z0, err)


@pytest.mark.parametrize("rotate", [False, True])
def test_recon_all_dezinger_then_phase_matches_reference(cuda, ref, rotate):
    """recon_all with outlier removal and Paganin phase retrieval (and
    projection rotation): the raw frames, darks and flats lose their outliers
    before dark/flat correction (proc_sino, proc_functions.py:146-148), then
    the chunk's phase retrieval and rotation, -log, filter, fourierrec.
    Against the restated chain (oracle dezinger, dark/flat, Paganin, rotate)
    feeding the reference's CUDA filter and fourierrec."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    nproj, nz, n, ncz = 90, 16, 128, 8
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=14)
    rng = np.random.default_rng(3)
    d32 = data.to(torch.int32)
    d32.view(-1)[torch.as_tensor(rng.integers(0, data.numel(), 300))] = 60000   # zingers
    data = d32.to(torch.uint16)
    opts = dict(rotate_proj_angle=1.5, rotate_proj_order=1) if rotate else {}
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=ncz, dezinger=3,
                      dezinger_threshold=5000, retrieve_phase_method="paganin",
                      pixel_size=0.65, propagation_distance=50.0, energy=20.0,
                      retrieve_phase_alpha=1e-3, **opts)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_all()
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    filt = ref.RefFilter(ne, nproj, ncz)
    rec = ref.RefFourierRec(n, nproj, ncz, torch.as_tensor(theta, device=cuda))
    for z0 in range(0, nz, ncz):
        sl = slice(z0, z0 + ncz)
        raw, dk, fl = (np_tomo.dezinger(a[:, sl].numpy(), 3, 5000.0) for a in (data, dark, flat))
        pre = np_tomo.darkflat(raw, dk, fl)
        pre = np_tomo.retrieve_phase(pre, "paganin", 0.65e-4, 5.0, 20.0, 1e-3)
        if rotate:
            pre = np_tomo.rotate_proj(pre, 1.5, 1)
        pre = np_tomo.minus_log(pre)
        d = torch.as_tensor(np.ascontiguousarray(pre.transpose(1, 0, 2)), device=cuda)
        d = ref.ref_fbp_filter_center(filt, d, wf, t, n / 2, torch.zeros(ncz, device=cuda), n, ne)
        theirs = torch.zeros((ncz, n, n), device=cuda)
        rec.backprojection(theirs, d)
        err = rel_l2(w.rec[sl].cpu(), theirs.cpu())
        assert err < 1e-4, (z0, err)


@pytest.mark.parametrize("algorithm", ["fourierrec", "linerec"])
def test_recon_try_with_phase_and_rotation_matches_reference(cuda, ref, algorithm):
    """recon_try with Paganin phase retrieval and projection rotation: the
    reference's recon_try runs proc_sino and proc_proj on the one-row slice
    (rec.py:224-225), so phase retrieval and rotation see images one row
    high; then the slice is tiled and filtered per centre shift."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    nproj, nz, n, ncz = 90, 8, 128, 4
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=15)
    global_vars.reset(reconstruction_type="try", reconstruction_algorithm=algorithm,
                      center_search_width=2.0, center_search_step=1.0, nsino="0.5",
                      nsino_per_chunk=ncz, retrieve_phase_method="paganin", pixel_size=0.65,
                      propagation_distance=50.0, energy=20.0, retrieve_phase_alpha=1e-3,
                      rotate_proj_angle=1.5)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_try()
    zs, shifts = int(params.id_slices[0]), params.shift_array
    assert len(w.tries) == len(shifts)
    sl = slice(zs, zs + 1)
    pre = np_tomo.darkflat(data[:, sl].numpy(), dark[:, sl].numpy(), flat[:, sl].numpy())
    pre = np_tomo.retrieve_phase(pre, "paganin", 0.65e-4, 5.0, 20.0, 1e-3)
    pre = np_tomo.minus_log(np_tomo.rotate_proj(pre, 1.5, 1))
    row = torch.as_tensor(np.ascontiguousarray(pre.transpose(1, 0, 2)), device=cuda)
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    filt = ref.RefFilter(ne, nproj, ncz)
    th = torch.as_tensor(theta, device=cuda)
    rec = (ref.RefFourierRec(n, nproj, ncz, th) if algorithm == "fourierrec"
           else ref.RefLineRec(th, nproj, nproj, ncz, ncz, n))
    for k in range(0, len(shifts), ncz):
        cnt = min(ncz, len(shifts) - k)
        sht = torch.zeros(ncz, device=cuda)
        sht[:cnt] = torch.as_tensor(shifts[k:k + cnt], device=cuda)
        d = ref.ref_fbp_filter_center(filt, row.repeat(ncz, 1, 1).contiguous(), wf, t, n / 2,
                                      sht, n, ne)
        theirs = torch.zeros((ncz, n, n), device=cuda)
        rec.backprojection(theirs, d)
        for kk in range(cnt):
            ours = w.tries[(zs, float(params.save_centers[k + kk]))].cpu()
            err = rel_l2(ours, theirs[kk].cpu())
            assert err < 1e-4, (k + kk, err)


@pytest.mark.parametrize("shape", [(4, 1024, 1024), (3, 700, 900)])
def test_phase_own_fft_matches_cufft(cuda, monkeypatch, shape):
    """Power-of-two padded sizes run on the library's own FFT (pairs of
    projections packed as one complex image, padding and crop fused into
    the row passes); the cuFFT R2C/C2R chain (TCB_PHASE_FFT set) computes
    the same filter.  An odd projection count leaves the last pair half
    empty."""
    _cases()
    from make_golden import phase_input
    x = phase_input(*shape, seed=13)
    args = ("paganin", 0.65e-4, 5.0, 20.0, 1e-3, 1500.0, 2e-4)
    own = _run(torch.as_tensor(x, device=cuda), *args, batch=4)
    monkeypatch.setenv("TCB_PHASE_FFT", "cufft")
    lib = _run(torch.as_tensor(x, device=cuda), *args, batch=4)
    err = rel_l2(own.cpu(), lib.cpu())
    print(f"phase own FFT vs cuFFT {shape}: {err:.2e}")
    assert err < 2e-6, err
