"""The reference's dtype 'float16' configuration through the drivers.

With dtype 'float16' the reference crops the projections to the centred
power-of-two width and shifts the centre (dataio/reader.py:155-165), takes a
power-of-two filter length (reconstruction/backproj_functions.py:52-54) and
runs its cfunc_*fp16 operators, writing float16 volumes.  Here the same
sizes and centre, fp16 output slices, fourierrec on the mixed-precision
(fp16 weights and values, fp32 accumulation) gridding, lprec and linerec
accumulating in fp32.  Budget: rel-L2 <= 2e-3 against the FP64 oracle (the
fp16 rounding of the output alone is ~3e-4)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _run(driver, data, dark, flat, theta, **opts):
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    from tomocupy_b200.rec_steps import GPURecSteps
    global_vars.reset(nsino_per_chunk=4, **opts)
    dt = torch.float16 if opts.get("dtype") == "float16" else torch.float32
    w = ArrayWriter(device="cuda", dtype=dt)
    r = ArrayReader(data, dark, flat, theta=theta)
    if driver == "all":
        GPURec(r, w).recon_all()
    else:
        GPURecSteps(r, w).recon_steps_all()
    return w.rec.cpu(), float(params.center), int(params.n), int(params.st_n)


@pytest.mark.parametrize("driver", ["all", "steps"])
def test_float16_fourierrec_crop_and_centre(cuda, driver):
    """ni = 300 columns -> the centred 256 (columns 22..277), centre 150 -> 128;
    the float16 volume against the FP64 oracle on those columns."""
    from oracle import np_tomo
    from tomocupy_b200 import synthetic
    nproj, nz, ni = 180, 4, 300
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, ni, seed=21)
    got, center, n, st = _run(driver, data, dark, flat, theta, dtype="float16")
    assert n == 256 and st == 22 and center == 128.0
    assert got.dtype == torch.float16 and tuple(got.shape) == (nz, n, n)
    d, dk, fl = (t[:, :, st:st + n].numpy() for t in (data, dark, flat))
    sino = np_tomo.minus_log(np_tomo.darkflat(d, dk, fl)).transpose(1, 0, 2).astype(np.float64)
    filt = np_tomo.fbp_filter_center(sino, np_tomo.calc_filter(4 * n, "parzen"), center, 0.0,
                                     np.float64)
    want = np_tomo.fourierrec(filt, theta, np.float64)
    err = rel_l2(got.float().numpy(), want)
    print(f"float16 fourierrec ({driver}) vs FP64: {err:.2e}")
    assert err < 2e-3, err


@pytest.mark.parametrize("algorithm", ["lprec", "linerec"])
def test_float16_lprec_linerec_match_float32(cuda, algorithm):
    """Power-of-two width (no crop): the float16 volume is the float32 one
    rounded to fp16."""
    from tomocupy_b200 import synthetic
    nproj, nz, n = 180, 4, 256
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=22)
    a, *_ = _run("all", data, dark, flat, theta, dtype="float16",
                 reconstruction_algorithm=algorithm)
    b, *_ = _run("all", data, dark, flat, theta, reconstruction_algorithm=algorithm)
    assert a.dtype == torch.float16
    assert torch.equal(a, b.to(torch.float16))
