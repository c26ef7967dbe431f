"""End-to-end GPU parity of the fused drivers against the reference's chain.

Workload: 16 rows x 360 angles over [0, pi) x 512 columns of uint16 frames
(seeded ellipsoid phantom, Poisson noise, 10 darks, 10 flats, centre 256),
Parzen filter, fourierrec; the reference chain is the reference's own CUDA
operators (oracle/_ref) behind a torch restatement of its CuPy glue.
"""
import numpy as np
import pytest
import torch

from conftest import TorchCuFFT, rel_l2

pytestmark = pytest.mark.gpu

N, NPROJ, NZ = 512, 360, 16


@pytest.fixture(scope="module")
def c1():
    from tomocupy_b200 import synthetic
    return synthetic.make_dataset(NPROJ, NZ, N, seed=0)


@pytest.fixture(scope="module")
def c1_thin():
    """The C1 geometry with a quarter of the densities (transmissions above
    ~8 %, no zero counts) and stripes.  Ring removal adds a correction to
    the normalised frames before -log; where a transmission is at or near
    zero (the C1 phantom has ~32 k such values per 8 rows), a last-bit
    difference between two float32 implementations of the correction moves
    a value across where(x <= 0, 1) or into log's steep region and changes
    the sinogram by O(1).  The ring-removal chains are compared on this
    well-conditioned phantom."""
    from tomocupy_b200 import synthetic
    return synthetic.make_dataset(NPROJ, NZ, N, seed=0, density_max=0.005, stripes=6)


def reference_chain(ref, data, dark, flat, theta, algorithm="fourierrec", ncz=8,
                    fbp="parzen", center=None, sht=None, stripe=None, flat_linear=False):
    from oracle import np_tomo
    dev = torch.device("cuda")
    P, nz, n = data.shape
    center = n / 2 if center is None else center
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, fbp), device=dev)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=dev)
    th = torch.as_tensor(theta, device=dev)
    filt = ref.RefFilter(ne, P, ncz)
    if algorithm == "fourierrec":
        rec = ref.RefFourierRec(n, P, ncz, th)
    elif algorithm == "lprec":
        from tomocupy_b200.reconstruction import lprec_grids as L
        ntheta, nrho = L.lp_sizes(n, P)
        A = L.create_adj(L.create_gl(n, P, ntheta, nrho))  # pinned by lprec_grids.npz
        rec = ref.RefLpRec(n, P, ncz, vars(A))
        center = center + 0.5  # BackprojFunctions (backproj_functions.py:70-71)
    else:
        rec = ref.RefLineRec(th, P, P, ncz, ncz, n)
    out = torch.zeros((nz, n, n), dtype=torch.float32, device=dev)
    for z0 in range(0, nz, ncz):
        # dark/flat in CuPy's float32 operation order (NumPy restatement,
        # bit-exact with the native kernel), -log with the device logf
        norm = np_tomo.darkflat_linear if flat_linear else np_tomo.darkflat
        d = norm(np.asarray(data[:, z0:z0 + ncz]), np.asarray(dark[:, z0:z0 + ncz]),
                 np.asarray(flat[:, z0:z0 + ncz]))
        # proc_sino: ring removal on the dark/flat corrected frames with the
        # oracle's restatements, which reproduce the reference's remove_stripe_ti
        # and remove_stripe_fw fixtures bit for bit (tests/test_stripe_*_cpu.py),
        # with their FFTs on cuFFT as cupy.fft runs them; then proc_proj: -log
        if stripe is not None and stripe[0] == "ti":
            d = np_tomo.remove_stripe_ti(d, stripe[1], stripe[2], fft=TorchCuFFT)
        elif stripe is not None:
            from tomocupy_b200.processing import wavelets
            sigma, wname, level = stripe
            d = np_tomo.remove_stripe_fw(d, sigma, level, wavelets.filter_bank(wname),
                                         fft=TorchCuFFT)
        d = torch.as_tensor(np.ascontiguousarray(d), device=dev)
        d = torch.where(d <= 0, torch.ones((), device=dev), d)
        d = torch.nan_to_num(-torch.log(d), nan=6.0, posinf=0.0, neginf=0.0)
        d = d.permute(1, 0, 2).contiguous()
        s = torch.zeros(ncz, device=dev) if sht is None else sht
        d = ref.ref_fbp_filter_center(filt, d, wf, t, center, s, n, ne)
        o = torch.zeros((ncz, n, n), dtype=torch.float32, device=dev)
        rec.backprojection(o, d)
        out[z0:z0 + ncz] = o
    torch.cuda.synchronize()
    return out.cpu()


def run_ours(data, dark, flat, theta, algorithm="fourierrec", ncz=8, host=True,
             dtype="float32", out_dtype="float32"):
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    global_vars.reset(reconstruction_algorithm=algorithm, nsino_per_chunk=ncz, dtype=dtype,
                      out_dtype=out_dtype)
    dev = "cpu" if host else "cuda"
    reader = ArrayReader(data.to(dev), dark.to(dev), flat.to(dev), theta=theta, pin=host)
    writer = ArrayWriter(device=dev, pin=host,
                         dtype=torch.float16 if out_dtype == "float16" else torch.float32)
    GPURec(reader, writer).recon_all()
    return writer.rec.cpu()


def test_c1_fourierrec_matches_reference(cuda, ref, c1):
    data, dark, flat, theta, _ = c1
    ours = run_ours(data, dark, flat, theta)
    theirs = reference_chain(ref, data, dark, flat, theta)
    err = rel_l2(ours, theirs)
    assert err < 1e-5, err


def test_c1_device_resident_equals_host_conveyor(cuda, c1):
    data, dark, flat, theta, _ = c1
    a = run_ours(data, dark, flat, theta, host=True)
    b = run_ours(data, dark, flat, theta, host=False)
    assert rel_l2(a, b) < 1e-6


def test_c1_chunk_size_invariance(cuda, c1):
    data, dark, flat, theta, _ = c1
    a = run_ours(data, dark, flat, theta, ncz=8)
    b = run_ours(data, dark, flat, theta, ncz=16)
    # the slice pairing changes with the chunk size; pairs are independent
    # reconstructions up to the reference's small real/imaginary crosstalk
    assert rel_l2(a, b) < 1e-4


def test_c1_linerec_matches_reference(cuda, ref, c1):
    data, dark, flat, theta, _ = c1
    d, dk, fl = data[:, :4], dark[:, :4], flat[:, :4]
    ours = run_ours(d, dk, fl, theta, algorithm="linerec", ncz=4)
    theirs = reference_chain(ref, d, dk, fl, theta, algorithm="linerec", ncz=4)
    err = rel_l2(ours, theirs)
    assert err < 1e-5, err


def test_c1_fw_ring_removal_pipeline(cuda, ref, c1_thin):
    """dark/flat -> fw ring removal (level 7, sym16) -> -log -> filter -> fourierrec."""
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    data, dark, flat, theta, _ = c1_thin
    d, dk, fl = data[:, :8], dark[:, :8], flat[:, :8]
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=8,
                      remove_stripe_method="fw", fw_sigma=1.0, fw_filter="sym16", fw_level=7)
    reader = ArrayReader(d, dk, fl, theta=theta, pin=True)
    writer = ArrayWriter(device="cpu", pin=True)
    GPURec(reader, writer).recon_all()
    theirs = reference_chain(ref, d, dk, fl, theta, ncz=8, stripe=(1.0, "sym16", 7))
    err = rel_l2(writer.rec, theirs)
    assert err < 1e-5, err


def test_c1_ti_ring_removal_pipeline(cuda, ref, c1_thin):
    """dark/flat -> Titarenko ring removal -> -log -> filter -> fourierrec, with a
    partial last chunk (12 rows in chunks of 8)."""
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    data, dark, flat, theta, _ = c1_thin
    d, dk, fl = data[:, :12], dark[:, :12], flat[:, :12]
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=8,
                      remove_stripe_method="ti", ti_beta=0.022, ti_mask=1)
    writer = ArrayWriter(device="cpu", pin=True)
    GPURec(ArrayReader(d, dk, fl, theta=theta, pin=True), writer).recon_all()
    theirs = reference_chain(ref, d[:, :8], dk[:, :8], fl[:, :8], theta, ncz=8,
                             stripe=("ti", 0.022, 1))
    err = rel_l2(writer.rec[:8], theirs)
    assert err < 1e-5, err


def test_c1_lprec_matches_reference(cuda, ref, c1):
    data, dark, flat, theta, _ = c1
    d, dk, fl = data[:, :4], dark[:, :4], flat[:, :4]
    ours = run_ours(d, dk, fl, theta, algorithm="lprec", ncz=4)
    theirs = reference_chain(ref, d, dk, fl, theta, algorithm="lprec", ncz=4)
    err = rel_l2(ours, theirs)
    assert err < 1e-5, err


def test_c1_error_vs_fp64_oracle(cuda, c1):
    """Accuracy statement: the fp32 path against the FP64 NumPy restatement."""
    from oracle import np_tomo
    data, dark, flat, theta, _ = c1
    d, dk, fl = data[:, :4], dark[:, :4], flat[:, :4]
    ours = run_ours(d, dk, fl, theta, ncz=4).numpy()
    sino = np_tomo.minus_log(np_tomo.darkflat(d.numpy(), dk.numpy(), fl.numpy()))
    sino = sino.transpose(1, 0, 2).astype(np.float64)
    wf = np_tomo.calc_filter(4 * N, "parzen")
    filt = np_tomo.fbp_filter_center(sino, wf, N / 2, 0.0, np.float64)
    want = np_tomo.fourierrec(filt, theta, np.float64)
    err = rel_l2(ours, want)
    assert err < 1e-4, err


def test_recon_try_matches_reference(cuda, ref, c1):
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    data, dark, flat, theta, _ = c1
    global_vars.reset(reconstruction_type="try", center_search_width=2.0,
                      center_search_step=0.5, nsino="0.5", nsino_per_chunk=4)
    reader = ArrayReader(data, dark, flat, theta=theta)
    writer = ArrayWriter(device="cuda")
    GPURec(reader, writer).recon_try()
    zs = int(params.id_slices[0])
    shifts = params.shift_array
    assert len(writer.tries) == len(shifts)
    # reference: the same slice tiled ncz times with per-slice centre shifts
    sl = data[:, zs:zs + 1].repeat(1, 4, 1)
    dk = dark[:, zs:zs + 1].repeat(1, 4, 1)
    fl = flat[:, zs:zs + 1].repeat(1, 4, 1)
    for k in range(0, len(shifts), 4):
        sht = torch.zeros(4, device="cuda")
        cnt = min(4, len(shifts) - k)
        sht[:cnt] = torch.as_tensor(shifts[k:k + cnt], device="cuda")
        theirs = reference_chain(ref, sl, dk, fl, theta, ncz=4, sht=sht)
        for kk in range(cnt):
            ours = writer.tries[(zs, float(params.save_centers[k + kk]))].cpu()
            err = rel_l2(ours, theirs[kk])
            assert err < 1e-5, (k + kk, err)


@pytest.mark.parametrize("algorithm", ["lprec", "linerec"])
def test_recon_try_lprec_linerec_match_reference(cuda, ref, c1, algorithm):
    """Try-centre reconstruction with the other backprojectors (the reference's
    recon_try runs whichever reconstruction_algorithm is set)."""
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    data, dark, flat, theta, _ = c1
    global_vars.reset(reconstruction_type="try", reconstruction_algorithm=algorithm,
                      center_search_width=2.0, center_search_step=0.5, nsino="0.5",
                      nsino_per_chunk=4)
    writer = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), writer).recon_try()
    zs, shifts = int(params.id_slices[0]), params.shift_array
    assert len(writer.tries) == len(shifts)
    sl, dk, fl = (t[:, zs:zs + 1].repeat(1, 4, 1) for t in (data, dark, flat))
    for k in range(0, len(shifts), 4):
        sht = torch.zeros(4, device="cuda")
        cnt = min(4, len(shifts) - k)
        sht[:cnt] = torch.as_tensor(shifts[k:k + cnt], device="cuda")
        theirs = reference_chain(ref, sl, dk, fl, theta, algorithm=algorithm, ncz=4, sht=sht)
        for kk in range(cnt):
            ours = writer.tries[(zs, float(params.save_centers[k + kk]))].cpu()
            err = rel_l2(ours, theirs[kk])
            assert err < 1e-5, (algorithm, k + kk, err)


@pytest.mark.parametrize("stripe", [("ti", 0.022, 1), (1.0, "sym16", 3)])
def test_recon_try_with_ring_removal_matches_reference(cuda, ref, c1_thin, stripe):
    """Try-centre sweep with ring removal of the slice (proc_sino inside the
    reference's recon_try, rec.py:224-226): Titarenko and Fourier-wavelet."""
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    data, dark, flat, theta, _ = c1_thin
    opts = (dict(remove_stripe_method="ti", ti_beta=stripe[1], ti_mask=stripe[2])
            if stripe[0] == "ti" else
            dict(remove_stripe_method="fw", fw_sigma=stripe[0], fw_filter=stripe[1],
                 fw_level=stripe[2]))
    global_vars.reset(reconstruction_type="try", center_search_width=2.0,
                      center_search_step=1.0, nsino="0.5", nsino_per_chunk=4, **opts)
    writer = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), writer).recon_try()
    zs, shifts = int(params.id_slices[0]), params.shift_array
    assert len(writer.tries) == len(shifts)
    sl, dk, fl = (t[:, zs:zs + 1].repeat(1, 4, 1) for t in (data, dark, flat))
    for k in range(0, len(shifts), 4):
        sht = torch.zeros(4, device="cuda")
        cnt = min(4, len(shifts) - k)
        sht[:cnt] = torch.as_tensor(shifts[k:k + cnt], device="cuda")
        theirs = reference_chain(ref, sl, dk, fl, theta, ncz=4, sht=sht, stripe=stripe)
        for kk in range(cnt):
            ours = writer.tries[(zs, float(params.save_centers[k + kk]))].cpu()
            err = rel_l2(ours, theirs[kk])
            assert err < 1e-5, (k + kk, err)


# --------------------------------------------------------------------------
# Mixed precision: split-fp16 tensor-core filter feeding the fp32 backprojectors.
# Budget: rel-L2 <= 1e-3 against the FP64 oracle of the same algorithm.
def _fp64_fourierrec(d, dk, fl, theta, n):
    from oracle import np_tomo
    sino = np_tomo.minus_log(np_tomo.darkflat(d.numpy(), dk.numpy(), fl.numpy()))
    sino = sino.transpose(1, 0, 2).astype(np.float64)
    wf = np_tomo.calc_filter(4 * n, "parzen")
    filt = np_tomo.fbp_filter_center(sino, wf, n / 2, 0.0, np.float64)
    return np_tomo.fourierrec(filt, theta, np.float64)


def test_c1_mixed_fourierrec_vs_fp64_oracle(cuda, c1):
    data, dark, flat, theta, _ = c1
    d, dk, fl = data[:, :4], dark[:, :4], flat[:, :4]
    mixed = run_ours(d, dk, fl, theta, ncz=4, dtype="mixed").numpy()
    fp32 = run_ours(d, dk, fl, theta, ncz=4).numpy()
    want = _fp64_fourierrec(d, dk, fl, theta, N)
    e_mixed, e_fp32 = rel_l2(mixed, want), rel_l2(fp32, want)
    assert e_mixed < 1e-3, e_mixed
    assert e_fp32 < 1e-4, e_fp32


@pytest.mark.parametrize("algorithm", ["linerec", "lprec"])
def test_c1_mixed_matches_fp32_path(cuda, c1, algorithm):
    data, dark, flat, theta, _ = c1
    d, dk, fl = data[:, :4], dark[:, :4], flat[:, :4]
    mixed = run_ours(d, dk, fl, theta, algorithm=algorithm, ncz=4, dtype="mixed")
    fp32 = run_ours(d, dk, fl, theta, algorithm=algorithm, ncz=4)
    err = rel_l2(mixed, fp32)
    assert err < 1e-4, err


def test_recon_try_mixed_matches_fp32(cuda, c1):
    """Per-centre filter kernels (one operator per slice) in the try sweep."""
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    data, dark, flat, theta, _ = c1
    res = {}
    for dtype in ("float32", "mixed"):
        global_vars.reset(reconstruction_type="try", center_search_width=2.0,
                          center_search_step=0.5, nsino="0.5", nsino_per_chunk=4, dtype=dtype)
        writer = ArrayWriter(device="cuda")
        GPURec(ArrayReader(data, dark, flat, theta=theta), writer).recon_try()
        res[dtype] = {k: v.cpu() for k, v in writer.tries.items()}
    assert res["float32"].keys() == res["mixed"].keys() and len(res["mixed"]) == 8
    # mixed precision grids with fp16 operands and keeps the oversampled grid
    # in fp16 (per-tile scales): within half the 1e-3 mixed budget of fp32
    for k in res["mixed"]:
        err = rel_l2(res["mixed"][k], res["float32"][k])
        assert err < 5e-4, (k, err)


def test_c1_mixed_fp16_output_vs_fp64_oracle(cuda, c1):
    """Mixed precision with fp16 output slices (half the device-to-host bytes)."""
    data, dark, flat, theta, _ = c1
    d, dk, fl = data[:, :4], dark[:, :4], flat[:, :4]
    out16 = run_ours(d, dk, fl, theta, ncz=4, dtype="mixed", out_dtype="float16")
    out32 = run_ours(d, dk, fl, theta, ncz=4, dtype="mixed")
    assert out16.dtype == torch.float16
    want = _fp64_fourierrec(d, dk, fl, theta, N)
    e16 = rel_l2(out16.float().numpy(), want)
    assert e16 < 1e-3, e16
    # the fp16 rounding of the output is the only difference
    assert rel_l2(out16.float(), out32) < 5e-4


def test_production_geometry_vs_fp64_oracle(cuda):
    """2048 columns x 1500 angles (the production geometry), 4 rows = 2 slice
    pairs: the fp32 path and the mixed-precision path against the FP64
    oracle of the same algorithm (fp32 <= 1e-4, mixed <= 1e-3), and mixed
    against fp32."""
    from tomocupy_b200 import synthetic
    n, nproj, nz = 2048, 1500, 4
    d, dk, fl, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=5)
    fp32 = run_ours(d, dk, fl, theta, ncz=nz, host=False).numpy()
    mixed = run_ours(d, dk, fl, theta, ncz=nz, host=False, dtype="mixed").numpy()
    want = _fp64_fourierrec(d, dk, fl, theta, n)
    e32, emix = rel_l2(fp32, want), rel_l2(mixed, want)
    print(f"2048x1500: fp32 vs FP64 {e32:.2e}, mixed vs FP64 {emix:.2e}, "
          f"mixed vs fp32 {rel_l2(mixed, fp32):.2e}")
    assert e32 < 1e-4, e32
    assert emix < 1e-3, emix


def test_c1_flat_linear_matches_reference(cuda, ref):
    """flat_linear (proc_functions.py:62-66: flats blended linearly over the
    angles from the means of the first and the last half) in the fused
    driver, 8 flats, against the restated normalisation feeding the
    reference's filter and fourierrec."""
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    d, dk, fl, theta, _ = synthetic.make_dataset(NPROJ, 8, N, seed=17, nflat=8)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=8,
                      flat_linear="True")
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(d, dk, fl, theta=theta), w).recon_all()
    theirs = reference_chain(ref, d, dk, fl, theta, ncz=8, flat_linear=True)
    err = rel_l2(w.rec.cpu(), theirs)
    assert err < 1e-5, err
