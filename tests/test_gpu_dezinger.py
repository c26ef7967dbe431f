"""GPU parity of the native outlier removal (tcb_dezinger) against fixtures
made by the reference's own remove_outliers: bit for bit (the window values
are exact in float, the sort network and the rank are the rank filter's),
on strided views and inside the fused pipeline."""
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import DEZINGER_CASES
    return DEZINGER_CASES


@pytest.mark.parametrize("i", range(5))
def test_dezinger_matches_reference_fixture(cuda, i):
    from tomocupy_b200.processing.proc_functions import dezinger
    g = np.load(ROOT / "tests" / "golden" / "dezinger.npz")
    dt, nf, nz, n, w, thr, seed = _cases()[i]
    x = torch.as_tensor(g[f"in_{i}"].astype(np.int32) if dt == "uint16" else g[f"in_{i}"])
    x = x.to(torch.uint16) if dt == "uint16" else x
    got = dezinger(x.to(cuda), w, thr)
    torch.cuda.synchronize()
    want = g[f"out_{i}"]
    assert np.array_equal(got.cpu().numpy().astype(want.dtype), want), i


def test_dezinger_strided_rows_and_widths(cuda):
    """A row slab of a larger stack (strided view) against the oracle, for
    every supported window size class."""
    from oracle import np_tomo
    from tomocupy_b200.processing.proc_functions import dezinger
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import dezinger_input
    full = dezinger_input("uint16", 40, 9, 70, seed=8)
    for w in (1, 2, 3, 5, 7, 9, 11):
        want = np_tomo.dezinger(full[:, 3:7], w, 400)
        src = torch.as_tensor(full.astype(np.int32)).to(torch.uint16).to(cuda)[:, 3:7]
        got = dezinger(src, w, 400).cpu().numpy().astype(np.uint16)
        assert np.array_equal(got, want), w


def test_fused_pipeline_with_dezinger(cuda, ref):
    """GPURec with dezinger 3 / threshold 500 (data, darks and flats cleaned,
    as proc_sino does) against the reference chain fed with frames cleaned by
    the oracle."""
    from oracle import np_tomo
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    from tomocupy_b200 import synthetic
    from test_gpu_pipeline import reference_chain
    nproj, nz, n = 120, 8, 128
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=5)
    rng = np.random.default_rng(0)
    d = data.numpy().copy()
    spikes = rng.random(d.shape) < 0.01
    d[spikes] = np.minimum(65535, d[spikes].astype(np.int64) + 8000).astype(np.uint16)
    d = torch.as_tensor(d.astype(np.int32)).to(torch.uint16)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=8, dezinger=3,
                      dezinger_threshold=500)
    w = ArrayWriter(device="cpu", pin=True)
    GPURec(ArrayReader(d, dark, flat, theta=theta, pin=True), w).recon_all()
    clean = [torch.as_tensor(np_tomo.dezinger(t.numpy(), 3, 500).astype(np.int32)).to(torch.uint16)
             for t in (d, dark, flat)]
    theirs = reference_chain(ref, *clean, theta, ncz=8)
    assert rel_l2(w.rec, theirs) < 1e-5
