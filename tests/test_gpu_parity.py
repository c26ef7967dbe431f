"""GPU parity of the native operators against the reference's own CUDA build.

The reference operators (oracle/_ref, compiled from the reference sources)
run on the same inputs through oracle.refglue.  Tolerances:
  * pre-processing: bit-exact (float32, same operation order);
  * filter: rel-L2 <= 1e-6 (same cuFFT transforms, own spectrum multiply);
  * fourierrec: rel-L2 <= 1e-5 (the reference accumulates with unordered
    atomics, ours in shared-memory tiles: summation order differs);
  * linerec: bit-identical (the reference's roundings written out).
"""
import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FR_TOL = 1e-5


def _theta(nproj, kind="uniform", seed=0):
    if kind == "uniform":
        return (np.arange(nproj) * np.pi / nproj).astype(np.float32)
    rng = np.random.default_rng(seed)
    return np.sort(rng.uniform(0, np.pi, nproj)).astype(np.float32)


# ------------------------------------------------------------------ prep
def test_prep_bit_exact(cuda):
    from oracle import np_tomo
    from tomocupy_b200 import synthetic
    from tomocupy_b200.processing.proc_functions import darkflat_stats, prep_rows
    data, dark, flat, _, _ = synthetic.make_dataset(90, 6, 200, seed=3)
    dd, dk, fl = data.to(cuda), dark.to(cuda), flat.to(cuda)
    d0, f0, _ = darkflat_stats(dk, fl)
    P, nz, n = data.shape
    out = torch.empty((nz, P, n), dtype=torch.float32, device=cuda)
    prep_rows(out, dd, d0, f0, darkflat=True, minus_log=False, out_zstride=P * n, out_pstride=n)
    want = np_tomo.darkflat(data.numpy(), dark.numpy(), flat.numpy()).transpose(1, 0, 2)
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    # -log: bit-exact against the device logf (torch.log); NumPy's log is a
    # different implementation (a few ulp)
    lg = torch.empty_like(out)
    prep_rows(lg, dd, d0, f0, darkflat=True, minus_log=True, out_zstride=P * n, out_pstride=n)
    x = torch.where(out <= 0, torch.ones((), device=cuda), out)
    tl = torch.nan_to_num(-torch.log(x), nan=6.0, posinf=0.0, neginf=0.0)
    np.testing.assert_array_equal(lg.cpu().numpy(), tl.cpu().numpy())
    np.testing.assert_array_max_ulp(lg.cpu().numpy(), np_tomo.minus_log(want), maxulp=4)


def test_prep_edge_cases(cuda):
    """Zero/negative normalised values, NaN (0/0) and +-inf follow nan_to_num(6, 0, 0)."""
    from tomocupy_b200.processing.proc_functions import prep_rows
    vals = torch.tensor([[[0.0, -1.0, float("nan"), float("inf"), 1e-30, 1.0, 2.0, 0.5]]],
                        device=cuda)
    out = torch.empty_like(vals)
    prep_rows(out, vals, darkflat=False, minus_log=True, out_zstride=8, out_pstride=8)
    got = out.cpu().numpy().ravel()
    want = np.array([0.0, 0.0, 6.0, 0.0, -np.log(np.float32(1e-30)), 0.0, -np.log(2.0),
                     -np.log(0.5)], dtype=np.float32)
    np.testing.assert_allclose(got, want, rtol=1e-6)


def test_flat_linear_matches_oracle(cuda):
    from oracle import np_tomo
    from tomocupy_b200 import synthetic
    from tomocupy_b200.processing.proc_functions import darkflat_stats, prep_rows
    data, dark, flat, _, _ = synthetic.make_dataset(40, 3, 96, seed=4, nflat=8)
    dd = data.to(cuda)
    d0, f0, f1 = darkflat_stats(dark.to(cuda), flat.to(cuda), flat_linear=True)
    P, nz, n = data.shape
    out = torch.empty((P, nz, n), dtype=torch.float32, device=cuda)
    prep_rows(out, dd, d0, f0, f1, darkflat=True, minus_log=False, flat_linear=True,
              out_zstride=n, out_pstride=nz * n)
    want = np_tomo.darkflat_linear(data.numpy(), dark.numpy(), flat.numpy())
    np.testing.assert_array_equal(out.cpu().numpy(), want)


# ------------------------------------------------------------------ filter
@pytest.mark.parametrize("nz,nproj,ne", [(2, 50, 512), (3, 90, 2048), (4, 33, 1000)])
def test_filter_vs_reference(cuda, ref, nz, nproj, ne):
    from tomocupy_b200 import cfunc_filter
    g = torch.randn((nz, nproj, ne), device=cuda)
    w = torch.randn((nz, ne // 2 + 1), dtype=torch.complex64, device=cuda)
    a = g.clone()
    cfunc_filter.cfunc_filter(nproj, nz, ne).filter(a, torch.view_as_real(w).contiguous(), None)
    b = g.clone()
    ref.RefFilter(ne, nproj, nz).filter(b, w)
    torch.cuda.synchronize()
    assert rel_l2(a.cpu(), b.cpu()) < 1e-6


def test_fbp_filter_center_vs_reference(cuda, ref):
    from tomocupy_b200 import global_vars
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.reconstruction.backproj_functions import BackprojFunctions
    global_vars.reset(reconstruction_algorithm="linerec", fbp_filter="shepp")
    n, nproj, ncz = 96, 40, 4
    params.n, params.nproj, params.ncz, params.nz = n, nproj, ncz, ncz
    params.center, params.centeri = 50.25, 50.25
    params.theta = _theta(nproj)
    bf = BackprojFunctions()
    data = torch.randn((ncz, nproj, n), device=cuda)
    sht = torch.tensor([0.0, 1.5, -3.25, 7.0], device=cuda)
    a = bf.fbp_filter_center(data.clone(), sht)
    rf = ref.RefFilter(bf.cl_filter.n, nproj, ncz)
    b = ref.ref_fbp_filter_center(rf, data.clone(), bf.wfilter, bf.t, params.center, sht, n,
                                  params.ne)
    torch.cuda.synchronize()
    assert rel_l2(a.cpu(), b.cpu()) < 1e-6


# ------------------------------------------------------------------ fourierrec
FR_CASES = [
    (128, 90, 2, "uniform"),
    (512, 360, 8, "uniform"),
    (200, 120, 3, "random"),   # 2n not a multiple of the tile: partial tiles
    (256, 401, 1, "random"),
    (2048, 150, 2, "uniform"),  # 2n = 4096: the production FFT length
    (2048, 1500, 4, "uniform"),  # the production geometry: 2048 columns x 1500 angles
    (4096, 64, 1, "random"),    # 2n = 8192: radix-16^3 x 2
]


@pytest.mark.parametrize("n,nproj,nz,kind", FR_CASES)
def test_fourierrec_dropin_vs_reference(cuda, ref, n, nproj, nz, kind):
    from tomocupy_b200 import cfunc_fourierrec
    theta = torch.as_tensor(_theta(nproj, kind), device=cuda)
    g = torch.randn((nz, nproj, n, 2), device=cuda)
    f_ours = torch.empty((nz, n, n, 2), device=cuda)
    ours = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
    ours.backprojection(f_ours, g.clone(), None)
    f_ref = torch.empty((nz, n, n, 2), device=cuda)
    L = ref.lib("fourierrec")
    h = L.ref_create(nproj, nz, n, theta.data_ptr())
    gr = g.clone()
    L.ref_backprojection(h, f_ref.data_ptr(), gr.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    L.ref_destroy(h)
    err = rel_l2(f_ours.cpu(), f_ref.cpu())
    assert err < FR_TOL, err


@pytest.mark.parametrize("n,nproj,nz", [(128, 60, 2), (256, 90, 3), (512, 100, 2),
                                        (1024, 64, 2), (2048, 40, 1), (4096, 24, 1)])
def test_fourierrec_own_fft_matches_cufft(cuda, monkeypatch, n, nproj, nz):
    """The own pruned inverse FFT (+ fused deapodization), rows first and
    columns first, with the largest and with one column per block, against
    cuFFT's pruned path."""
    from tomocupy_b200 import cfunc_fourierrec
    theta = torch.as_tensor(_theta(nproj, "random"), device=cuda)
    g = torch.randn((nz, nproj, n, 2), device=cuda)
    out = {}
    for mode, cpc in (("cufft", None), ("own", None), ("own", "1"), ("own_cf", None),
                      ("own_cf", "2")):
        monkeypatch.setenv("TCB_FOURIERREC_FFT", mode)
        if cpc is None:
            monkeypatch.delenv("TCB_FOURIERREC_FFT_CPC", raising=False)
        else:
            monkeypatch.setenv("TCB_FOURIERREC_FFT_CPC", cpc)
        op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
        f = torch.full((nz, n, n, 2), float("nan"), device=cuda)
        op.backprojection(f, g.clone(), None)
        torch.cuda.synchronize()
        out[(mode, cpc)] = f.cpu()
        op.free()
    want = out.pop(("cufft", None))
    for key, got in out.items():
        err = rel_l2(got, want)
        assert err < 1e-6, (key, err)


@pytest.mark.parametrize("n,nproj,nz", [(128, 90, 2), (200, 120, 3), (512, 360, 16),
                                        (256, 180, 20), (2048, 64, 8), (256, 100, 40)])
def test_fourierrec_tensor_gridding_vs_fp32(cuda, n, nproj, nz):
    """Mixed-precision gridding (fp16 weights and values on tcgen05, fp32
    accumulation, 32 slice pairs per CTA) against the fp32 gridding: partial
    tiles (n = 200), pair counts that are not a multiple of 32, more than 32
    pairs (two groups)."""
    from tomocupy_b200 import _lib, cfunc_fourierrec
    theta = torch.as_tensor(_theta(nproj, "random"), device=cuda)
    g = torch.randn((nz, nproj, n, 2), device=cuda) * 100.0
    out = {}
    for mode in (_lib.GRID_FP32, _lib.GRID_TENSOR):
        op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
        op.set_gridding(mode)
        f = torch.full((nz, n, n, 2), float("nan"), device=cuda)
        op.backprojection(f, g.clone(), None)
        torch.cuda.synchronize()
        assert not op.timed_out()
        out[mode] = f.cpu()
        op.free()
    assert torch.isfinite(out[_lib.GRID_TENSOR]).all()
    err = rel_l2(out[_lib.GRID_TENSOR], out[_lib.GRID_FP32])
    print(f"tensor gridding n={n} nz={nz}: rel-L2 vs fp32 {err:.2e}")
    assert err < 1e-3, err


def test_fourierrec_backprojection_slices_matches_dropin(cuda):
    from tomocupy_b200 import cfunc_fourierrec
    n, nproj, nz = 128, 64, 2
    theta = torch.as_tensor(_theta(nproj), device=cuda)
    op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
    g = torch.randn((nz, nproj, n, 2), device=cuda)
    fc = torch.empty((nz, n, n, 2), device=cuda)
    op.backprojection(fc, g.clone(), None)
    fs = torch.empty((2 * nz, n, n), device=cuda)
    op.backprojection_slices(fs, g.clone(), None)
    torch.cuda.synchronize()
    # two runs differ only by the order of shared-memory accumulation
    assert rel_l2(fs[:nz].cpu(), fc[..., 0].cpu()) < 1e-6
    assert rel_l2(fs[nz:].cpu(), fc[..., 1].cpu()) < 1e-6


@pytest.mark.parametrize("n,nproj,nz", [(256, 180, 2), (512, 360, 40)])
def test_fourierrec_deterministic(cuda, n, nproj, nz):
    """Both gridding modes sum in a fixed order (registers or TMEM, no atomics)
    and every other stage is a fixed sequence of operations: two runs are
    bit-identical."""
    from tomocupy_b200 import _lib, cfunc_fourierrec
    theta = torch.as_tensor(_theta(nproj), device=cuda)
    g = torch.randn((nz, nproj, n, 2), device=cuda)
    for mode in (_lib.GRID_FP32, _lib.GRID_TENSOR):
        op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
        op.set_gridding(mode)
        outs = []
        for _ in range(2):
            f = torch.empty((nz, n, n, 2), device=cuda)
            op.backprojection(f, g.clone(), None)
            outs.append(f.cpu())
        assert not op.timed_out()
        op.free()
        assert torch.equal(outs[0], outs[1]), mode


def test_fourierrec_fp16_vs_fp64(cuda):
    from oracle import np_tomo
    from tomocupy_b200 import cfunc_fourierrecfp16
    n, nproj, nz = 128, 90, 2
    th = _theta(nproj)
    theta = torch.as_tensor(th, device=cuda)
    rng = np.random.default_rng(1)
    g = rng.standard_normal((nz, nproj, n)) + 1j * rng.standard_normal((nz, nproj, n))
    gh = torch.view_as_real(torch.as_tensor(g.astype(np.complex64))).to(torch.float16).to(cuda)
    op = cfunc_fourierrecfp16.cfunc_fourierrec(nproj, nz, n, theta)
    f = torch.empty((nz, n, n, 2), dtype=torch.float16, device=cuda)
    op.backprojection(f, gh.contiguous(), None)
    torch.cuda.synchronize()
    want = np_tomo.fourierrec_pairs(g, th, n, np.float64)
    got = torch.view_as_complex(f.float().contiguous()).cpu().numpy()
    assert rel_l2(got, want) < 2e-3


def test_fourierrec_vs_numpy_oracle(cuda):
    """The float32 NumPy restatement agrees with the native operator (pins the oracle)."""
    from oracle import np_tomo
    from tomocupy_b200 import cfunc_fourierrec
    n, nproj, nz = 128, 90, 2
    th = _theta(nproj)
    rng = np.random.default_rng(2)
    g = (rng.standard_normal((nz, nproj, n)) + 1j * rng.standard_normal((nz, nproj, n))).astype(
        np.complex64)
    op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, torch.as_tensor(th, device=cuda))
    f = torch.empty((nz, n, n, 2), device=cuda)
    op.backprojection(f, torch.view_as_real(torch.as_tensor(g)).to(cuda).contiguous(), None)
    torch.cuda.synchronize()
    got = torch.view_as_complex(f.contiguous()).cpu().numpy()
    assert rel_l2(got, np_tomo.fourierrec_pairs(g, th, n, np.float32)) < 1e-4
    assert rel_l2(got, np_tomo.fourierrec_pairs(g, th, n, np.float64)) < 1e-4


# ------------------------------------------------------------------ linerec
def _linerec_pair(cuda, ref, n, nproj, nz, ncz, mode, dtype="float32"):
    from tomocupy_b200.reconstruction.linerec import LineRec
    theta = torch.as_tensor(_theta(nproj), device=cuda)
    tdt = torch.float16 if dtype == "float16" else torch.float32
    data = torch.randn((nz, nproj, n), device=cuda).to(tdt)
    ours = LineRec(theta, nproj, nproj, nz, ncz, n, dtype)
    theirs = ref.RefLineRec(theta, nproj, nproj, nz, ncz, n, dtype)
    fa = torch.zeros((ncz, n, n), dtype=tdt, device=cuda)
    fb = torch.zeros((ncz, n, n), dtype=tdt, device=cuda)
    if mode == "full":
        ours.backprojection(fa, data)
        theirs.backprojection(fb, data)
    elif mode == "lamino":
        ours.backprojection(fa, data, None, theta, lamino_angle=20.0, sz=3)
        theirs.backprojection(fb, data, None, theta, lamino_angle=20.0, sz=3)
    elif mode == "try":
        sh = torch.linspace(-3, 3, ncz, device=cuda)
        ours.backprojection_try(fa, data, sh, None, theta, lamino_angle=0.0, sz=nz // 2)
        theirs.backprojection_try(fb, data, sh, None, theta, lamino_angle=0.0, sz=nz // 2)
    else:
        sh = torch.linspace(-2, 2, ncz, device=cuda)
        ours.backprojection_try_lamino(fa, data, sh, None, theta, lamino_angle=25.0, sz=nz // 2)
        theirs.backprojection_try_lamino(fb, data, sh, None, theta, lamino_angle=25.0, sz=nz // 2)
    torch.cuda.synchronize()
    return fa.float().cpu(), fb.float().cpu()


@pytest.mark.parametrize("phi_deg,n,nproj,nz,ncz,sz", [(90.0, 256, 181, 12, 7, 2),
                                                       (90.0, 2048, 70, 8, 8, 0),
                                                       (110.0, 200, 90, 16, 6, 5)])
def test_linerec_tma_staging_is_bit_identical(cuda, monkeypatch, phi_deg, n, nproj, nz, ncz, sz):
    """The float32 full backprojection with its sinogram boxes staged by TMA
    (two stages, mbarrier waits) sums the same values in the same order as
    the plain staging: identical results, with a partial angle chunk, a
    partial slice group, the full 2048 width, and a tilted (laminography)
    geometry whose footprints leave the boxes."""
    from tomocupy_b200 import cfunc_linerec
    theta = torch.as_tensor(_theta(nproj, "random", seed=5), device=cuda)
    g = torch.randn((nz, nproj, n), device=cuda)
    out = []
    for tma in ("1", "0"):
        monkeypatch.setenv("TCB_LINEREC_TMA", tma)
        op = cfunc_linerec.cfunc_linerec(nproj, nz, n, nproj, ncz)
        f = torch.full((ncz, n, n), 0.5, device=cuda)
        op.backprojection(f, g, theta, math.radians(phi_deg), sz, None)
        torch.cuda.synchronize()
        assert not op.timed_out()
        op.free()
        out.append(f.cpu())
    assert torch.equal(out[0], out[1])


@pytest.mark.parametrize("mode", ["full", "lamino", "try", "try_lamino"])
def test_linerec_vs_reference(cuda, ref, mode):
    """float32: the reference build's u, v, truncations, weights and
    per-voxel angle sums in the same roundings and order: bit-identical."""
    nz = 4 if mode == "full" else 16
    ncz = 4
    a, b = _linerec_pair(cuda, ref, 96, 60, nz, ncz, mode)
    assert torch.equal(a, b), rel_l2(a, b)


def test_linerec_fp16_storage_fp32_accumulation(cuda, ref):
    """fp16 buffers, fp32 sums: closer to the fp32 result than the reference's fp16 sums."""
    a32, b32 = _linerec_pair(cuda, ref, 96, 60, 4, 4, "full", "float32")
    torch.manual_seed(0)
    a16, b16 = _linerec_pair(cuda, ref, 96, 60, 4, 4, "full", "float16")
    assert rel_l2(a16, b16) < 5e-2  # same inputs rounded to fp16 (different draws)
