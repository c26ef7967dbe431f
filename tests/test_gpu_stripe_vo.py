"""Vo's all-stripe ring removal on the GPU (tcb_stripe_vo_*) against the
reference's remove_all_stripe: the fixtures it produced (tests/golden/
vo_stripe.npz) and the NumPy restatement pinned to them, on larger chunks with
the default windows, and inside the fused driver.  Sorts, medians and the
interpolation weights are exact; the float32 means and sums of the stripe
detection add in another order, hence rel-L2 <= 1e-5 rather than equality."""
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import VO_CASES, vo_input
    return VO_CASES, vo_input


@pytest.mark.parametrize("i", range(3))
def test_vo_matches_reference_fixture(cuda, i):
    from tomocupy_b200.processing.remove_stripe import remove_all_stripe
    cases, _ = _cases()
    nproj, nz, ni, snr, la, sm, seed = cases[i]
    g = np.load(ROOT / "tests" / "golden" / "vo_stripe.npz")
    got = remove_all_stripe(torch.as_tensor(g[f"in_{i}"], device=cuda), snr, la, sm)
    torch.cuda.synchronize()
    err = rel_l2(got.cpu().numpy(), g[f"out_{i}"])
    assert err < 1e-5, (i, err)


@pytest.mark.parametrize("nproj,nz,ni", [(360, 4, 512), (1500, 2, 1024)])
def test_vo_default_windows_vs_oracle(cuda, nproj, nz, ni):
    from oracle import np_tomo
    from tomocupy_b200.processing.remove_stripe import remove_all_stripe
    _, vo_input = _cases()
    data = vo_input(nproj, nz, ni, seed=nproj)
    got = remove_all_stripe(torch.as_tensor(data, device=cuda), 3.0, 61, 21)
    torch.cuda.synchronize()
    want = np_tomo.remove_all_stripe(data, 3.0, 61, 21)
    err = rel_l2(got.cpu().numpy(), want)
    assert err < 1e-5, err


def test_vo_fused_driver_matches_reference_chain(cuda, ref):
    """dark/flat -> Vo's ring removal -> -log -> filter -> fourierrec in
    GPURec.recon_all against the restated ring removal feeding the
    reference's filter and fourierrec (a phantom without zero transmissions,
    as the other ring-removal chains)."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    nproj, nz, n = 360, 8, 512
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=4,
                                                        density_max=0.005, stripes=8)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=8,
                      remove_stripe_method="vo-all")
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_all()
    pre = np_tomo.darkflat(data.numpy(), dark.numpy(), flat.numpy())
    pre = np_tomo.minus_log(np_tomo.remove_all_stripe(pre, 3.0, 61, 21))
    ne = 4 * n
    wf = torch.as_tensor(np_tomo.calc_filter(ne, "parzen"), device=cuda)
    t = torch.as_tensor(np_tomo.rfftfreq32(ne), device=cuda)
    d = torch.as_tensor(np.ascontiguousarray(pre.transpose(1, 0, 2)), device=cuda)
    d = ref.ref_fbp_filter_center(ref.RefFilter(ne, nproj, nz), d, wf, t, n / 2,
                                  torch.zeros(nz, device=cuda), n, ne)
    theirs = torch.zeros((nz, n, n), device=cuda)
    ref.RefFourierRec(n, nproj, nz, torch.as_tensor(theta, device=cuda)).backprojection(theirs, d)
    err = rel_l2(w.rec.cpu(), theirs.cpu())
    assert err < 1e-5, err
