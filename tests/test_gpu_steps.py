"""GPU checks of the step-wise driver (GPURecSteps.recon_steps_all) against the
reference chain: laminography with linerec accumulates over angle chunks in
the reference (backproj_parallel.py:94-168) with the projections filtered
per chunk; here everything is filtered once and backprojected over all
angles (same sum, grouped differently): rel-L2 <= 1e-5."""
import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _data(nproj, nz, n, seed=5):
    from tomocupy_b200 import synthetic
    return synthetic.make_dataset(nproj, nz, n, seed=seed,
                                  theta=(np.arange(nproj) * 2 * np.pi / nproj).astype(np.float32))


def test_steps_lamino_linerec_full_matches_reference(cuda, ref):
    from oracle import np_tomo
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec_steps import GPURecSteps
    nproj, nz, n, tilt = 40, 16, 64, 20.0
    data, dark, flat, theta, _ = _data(nproj, nz, n)
    global_vars.reset(reconstruction_algorithm="linerec", reconstruction_type="full",
                      lamino_angle=tilt, nsino_per_chunk=4, nproj_per_chunk=8,
                      lamino_end_row=8, fbp_filter="parzen")
    reader = ArrayReader(data, dark, flat, theta=theta)
    writer = ArrayWriter(device="cuda")
    ours = GPURecSteps(reader, writer).recon_steps_all().cpu()
    # reference: per row chunk, per angle chunk: filter + accumulate
    dev = torch.device("cuda")
    d = ref.ref_darkflat_minus_log(data.to(dev), dark.to(dev), flat.to(dev))  # [P, nz, n]
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=dev)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=dev)
    th = torch.as_tensor(theta, device=dev)
    ncproj, ncz, rh = 8, 4, params.rh
    filt = ref.RefFilter(ne, ncproj, nz)
    lr = ref.RefLineRec(th, nproj, ncproj, nz, ncz, n)
    vol = torch.zeros((rh, n, n), device=dev)
    for r0 in range(0, rh, ncz):
        f = torch.zeros((ncz, n, n), device=dev)
        for p0 in range(0, nproj, ncproj):
            d0 = d[p0:p0 + ncproj].permute(1, 0, 2).contiguous()  # [nz, ncproj, n]
            d0 = ref.ref_fbp_filter_center(filt, d0, wf, t, params.center, 0.0, n, ne)
            lr.backprojection(f, d0, None, th[p0:p0 + ncproj].contiguous(), tilt, r0)
        vol[r0:r0 + ncz] = f[:min(ncz, rh - r0)]
    torch.cuda.synchronize()
    err = rel_l2(ours, vol.cpu())
    assert err < 1e-5, err


def test_steps_lamino_fourierrec_matches_reference(cuda, ref):
    """recon_steps_all dispatches laminography + fourierrec to the Fourier
    chain: the reference's rec_lam (its operators behind the restated glue)
    on the same dark/flat-corrected, -log projections."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import args, params
    from tomocupy_b200.rec_steps import GPURecSteps
    nproj, nz, n, tilt = 48, 64, 64, 30.0
    data, dark, flat, theta, _ = _data(nproj, nz, n)
    global_vars.reset(reconstruction_algorithm="fourierrec", reconstruction_type="full",
                      lamino_angle=tilt, nsino_per_chunk=8, nproj_per_chunk=8,
                      lamino_end_row=32)
    u = GPURecSteps(ArrayReader(data, dark, flat, theta=theta),
                    ArrayWriter(device="cuda")).recon_steps_all().cpu()
    assert tuple(u.shape) == (32, n, n) and torch.isfinite(u).all()
    dev = torch.device("cuda")
    d = ref.ref_darkflat_minus_log(data.to(dev), dark.to(dev), flat.to(dev))  # [P, nz, n]
    wf = torch.as_tensor(np_tomo.calc_filter(4 * n, args.fbp_filter), device=dev)
    theirs = ref.ref_rec_lam(d.contiguous(), torch.as_tensor(theta, device=dev), params.center,
                             tilt, params.rh, wf, nthetac=8, dethc=8, n1c=8).cpu()
    err = rel_l2(u, theirs)
    assert err < 1e-5, err
