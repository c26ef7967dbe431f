"""Try-centre sweeps (TryCenterSweep): CUDA-graph replay, mixed precision per
centre against the FP64 oracle, and the autotuner.

Parity of the fp32 sweep with the reference's own try chain is covered by
tests/test_gpu_pipeline.py::test_recon_try_matches_reference (GPURec.recon_try
runs on TryCenterSweep).
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from tomocupy_b200.trycenter import chunk_shifts


def test_chunk_shifts_pads_the_last_chunk():
    sh = chunk_shifts(np.arange(10, dtype=np.float32) * 0.5, 4)
    assert sh.shape == (3, 4)
    assert np.array_equal(sh.reshape(-1)[:10], np.arange(10) * 0.5)
    assert np.all(sh.reshape(-1)[10:] == 0)
    assert chunk_shifts([], 4).shape == (1, 4)


N, P, Z = 256, 180, 2


@pytest.fixture(scope="module")
def one_slice():
    from tomocupy_b200 import synthetic
    data, dark, flat, theta, _ = synthetic.make_dataset(P, Z, N, seed=5)
    return data[:, 1:2].contiguous(), dark[:, 1:2].contiguous(), flat[:, 1:2].contiguous(), theta


def _sweep(one_slice, precision, shifts, ncz=4, pairs=0, graph=True):
    from tomocupy_b200.processing.proc_functions import darkflat_stats
    from tomocupy_b200.trycenter import TryCenterSweep
    d, dk, fl, theta = one_slice
    d0, f0, _ = darkflat_stats(dk.cuda(), fl.cuda())
    sw = TryCenterSweep(N, P, theta, N / 2, shifts, "parzen", precision, ncz, pairs)
    sw.load(d.cuda(), d0, f0)
    if graph:
        sw.capture()
    return sw, sw.run().cpu().clone()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["float32", "mixed"])
def test_graph_replay_equals_eager(cuda, one_slice, precision):
    shifts = np.arange(-5, 5) * 0.75
    _, eager = _sweep(one_slice, precision, shifts, graph=False)
    sw, graph = _sweep(one_slice, precision, shifts, graph=True)
    assert torch.equal(eager, graph)
    # a second replay after reloading the same slice gives the same images
    again = sw.run().cpu()
    assert torch.equal(again, graph)


@pytest.mark.gpu
def test_mixed_sweep_vs_fp64_oracle_per_center(cuda, one_slice):
    from oracle import np_tomo
    from tomocupy_b200.trycenter import per_center_errors
    shifts = np.array([-3.0, -1.5, -0.375, 0.0, 1.125, 2.5])
    _, mixed = _sweep(one_slice, "mixed", shifts)
    _, fp32 = _sweep(one_slice, "float32", shifts)
    d, dk, fl, theta = one_slice
    sino = np_tomo.minus_log(np_tomo.darkflat(d.numpy(), dk.numpy(), fl.numpy()))
    sino = sino.transpose(1, 0, 2).astype(np.float64)  # [1, P, N]
    wf = np_tomo.calc_filter(4 * N, "parzen")
    filt = np.concatenate([np_tomo.fbp_filter_center(sino, wf, N / 2, s, np.float64)
                           for s in shifts])
    want = torch.as_tensor(np_tomo.fourierrec(filt, theta, np.float64))
    rel_m, max_m = per_center_errors(mixed, want)
    rel_f, _ = per_center_errors(fp32, want)
    assert rel_m.max() < 1e-3, rel_m
    assert rel_f.max() < 1e-4, rel_f
    assert np.all(np.isfinite(max_m))


@pytest.mark.gpu
def test_autotune_picks_a_candidate_with_identical_results(cuda, one_slice, tmp_path):
    from tomocupy_b200.processing.proc_functions import darkflat_stats
    from tomocupy_b200.trycenter import autotune
    d, dk, fl, theta = one_slice
    d0, f0, _ = darkflat_stats(dk.cuda(), fl.cuda())
    shifts = np.arange(8) * 0.5
    cache = tmp_path / "tune.json"
    res = autotune(N, P, theta, N / 2, shifts, d.cuda(), d0, f0, precision="float32",
                   candidates=[(4, 2), (8, 4)], cache_file=cache)
    assert (res["ncz"], res["pairs_per_block"]) in [(4, 2), (8, 4)]
    assert len(res["table"]) == 2 and cache.exists()
    _, a = _sweep(one_slice, "float32", shifts, ncz=res["ncz"], pairs=res["pairs_per_block"])
    _, b = _sweep(one_slice, "float32", shifts, ncz=4, pairs=0)
    # pair packing differs with the chunk size: independent reconstructions up
    # to the small real/imaginary crosstalk of the reference algorithm
    assert rel_l2(a, b) < 1e-4
