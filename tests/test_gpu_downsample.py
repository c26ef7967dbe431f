"""GPU parity of binning (tcb_downsample) against fixtures made by the
reference's own utils.downsample (bit for bit: the same float32 pairwise
order), and of a binned reconstruction through GPURec against the
reference's CUDA build fed with frames binned by the restatement."""
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu


def _cases():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import DOWNSAMPLE_CASES
    return DOWNSAMPLE_CASES


@pytest.mark.parametrize("i", range(4))
def test_downsample_matches_reference_fixture(cuda, i):
    from tomocupy_b200.processing.proc_functions import downsample
    k, zr, nr, b, integer, seed = _cases()[i]
    g = np.load(ROOT / "tests" / "golden" / "downsample.npz")
    x = torch.as_tensor(g[f"in_{i}"], device=cuda)
    got = downsample(x, b).cpu().numpy()
    assert np.array_equal(got, g[f"out_{i}"])


def test_downsample_uint16_view(cuda):
    """uint16 frames (exact integer sums) from a strided row slab."""
    from oracle import np_tomo
    from tomocupy_b200.processing.proc_functions import downsample
    rng = np.random.default_rng(3)
    raw = rng.integers(0, 65536, (5, 20, 48)).astype(np.uint16)
    src = torch.as_tensor(raw.astype(np.int32)).to(torch.uint16).to(cuda)[:, 4:16]
    got = downsample(src, 2).cpu().numpy()
    assert np.array_equal(got, np_tomo.downsample(raw[:, 4:16].astype(np.float32), 2))


def test_binned_reconstruction_matches_reference_chain(cuda, ref):
    from oracle import np_tomo
    from tomocupy_b200 import global_vars, synthetic
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.global_vars import params
    from tomocupy_b200.rec import GPURec
    from test_gpu_pipeline import reference_chain
    nproj, nz, n = 120, 16, 256
    data, dark, flat, theta, _ = synthetic.make_dataset(nproj, nz, n, seed=7)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=4, binning=1)
    w = ArrayWriter(device="cuda")
    GPURec(ArrayReader(data, dark, flat, theta=theta), w).recon_all()
    assert (params.nz, params.n) == (nz // 2, n // 2)
    binned = [torch.as_tensor(np_tomo.downsample(t.numpy().astype(np.float32), 1))
              for t in (data, dark, flat)]
    theirs = reference_chain(ref, *binned, theta, ncz=4, center=params.center)
    err = rel_l2(w.rec.cpu(), theirs)
    assert err < 1e-5, err
