"""Tensor-core filter: the Toeplitz statement of the filter chain (CPU) and
the tcgen05 GEMM against the FP64 oracle and the fp32 cuFFT path (GPU).

The operator identity is exact algebra (edge pad -> circular convolution ->
crop == one n x n matrix), so on the CPU it is checked to float64 round-off
against the oracle's FP64 fbp_filter_center.  On the GPU the split-fp16
GEMM (22-bit operands, fp32 accumulation over K = 3n) must agree with the
FP64 oracle within rel-L2 5e-5.  Measured on B200: 2e-6 (n=256) to 1.8e-5
(n=2048); the error grows with n because the ramp filter's output is a small
difference of large partial sums accumulated over K.  That is 50x inside the
1e-3 budget of the mixed-precision path.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

from oracle import np_tomo
from tomocupy_b200.reconstruction.tcfilter import (impulse_responses, split16,
                                                   toeplitz_operator)


def _rows(nz, P, n, seed=0):
    rng = np.random.default_rng(seed)
    # smooth sinogram-like rows (large DC, structure) plus noise
    x = np.linspace(-1, 1, n)
    base = np.clip(1 - x[None, None, :] ** 2, 0, None) * rng.uniform(0.5, 3, (nz, P, 1))
    return (base + 0.01 * rng.standard_normal((nz, P, n))).astype(np.float32)


@pytest.mark.parametrize("name,n,center,sht", [("parzen", 64, 32.0, 0.0),
                                               ("shepp", 96, 40.25, 1.5),
                                               ("ramp", 128, 70.0, -2.375)])
def test_toeplitz_operator_equals_fp64_filter_chain(name, n, center, sht):
    ne = 4 * n
    wf = np_tomo.calc_filter(ne, name)
    rows = _rows(1, 5, n)
    want = np_tomo.fbp_filter_center(rows.astype(np.float64), wf, center, sht, np.float64)
    hz = impulse_responses(wf, ne, n, center, sht)[0]
    T = toeplitz_operator(hz, n, ne // 2 - n // 2)
    got = rows[0].astype(np.float64) @ T.T
    assert np.abs(got - want[0]).max() <= 1e-10 * np.abs(want).max()


def test_impulse_responses_batch_matches_single():
    n, ne = 64, 256
    wf = np_tomo.calc_filter(ne, "shepp")
    shs = np.array([0.0, 0.5, -1.25])
    batch = impulse_responses(wf, ne, n, 30.0, shs)
    for k, s in enumerate(shs):
        assert np.array_equal(batch[k], impulse_responses(wf, ne, n, 30.0, s)[0])


def test_split16_reconstructs_fp32():
    x = torch.as_tensor(_rows(2, 3, 64))
    hi, lo = split16(x)
    assert hi.dtype == torch.float16 and lo.dtype == torch.float16
    err = (hi.float() + lo.float() - x).abs()
    assert float(err.max()) <= 2.0 ** -21 * float(x.abs().max())


@pytest.mark.gpu
@pytest.mark.parametrize("n,P,nz,name,center", [(512, 360, 4, "parzen", 256.0),
                                                (2048, 150, 2, "shepp", 1023.0),
                                                (320, 77, 3, "ramp", 150.5)])
def test_tc_filter_vs_fp64_oracle(cuda, n, P, nz, name, center):
    from tomocupy_b200.reconstruction.tcfilter import TCFilter
    ne = 4 * n
    wf = np_tomo.calc_filter(ne, name)
    rows = _rows(nz, P, n, seed=n)
    want = np_tomo.fbp_filter_center(rows.astype(np.float64), wf, center, 0.0, np.float64)
    x = torch.as_tensor(rows, device="cuda")
    hi, lo = split16(x)
    f = TCFilter(n, P, nz)
    f.set_kernels(wf, ne, center, 0.0)
    out = torch.full((nz, P, n), float("nan"), device="cuda")
    f.apply(hi, lo, out)
    torch.cuda.synchronize()
    assert not f.timed_out()
    err = rel_l2(out.cpu().double(), torch.as_tensor(want))
    assert err < 5e-5, err


@pytest.mark.gpu
def test_tc_filter_matches_fp32_cufft_filter(cuda):
    """Against the drop-in fp32 chain (edge pad, cuFFT R2C, x w, C2R, crop)."""
    from tomocupy_b200.reconstruction.backproj_functions import phase_weights, rfftfreq32
    from tomocupy_b200.reconstruction.fbp_filter import FBPFilter
    from tomocupy_b200.reconstruction.tcfilter import TCFilter
    n, P, nz, center = 1024, 200, 4, 511.0
    ne = 4 * n
    pad = ne // 2 - n // 2
    wf = np_tomo.calc_filter(ne, "shepp")
    x = torch.as_tensor(_rows(nz, P, n, seed=3), device="cuda")
    tmp = torch.empty((nz, P, ne), device="cuda")
    tmp[:, :, pad:pad + n] = x
    tmp[:, :, :pad] = x[:, :, :1]
    tmp[:, :, pad + n:] = x[:, :, -1:]
    w = phase_weights(torch.as_tensor(wf, device="cuda"), rfftfreq32(ne, "cuda"), center,
                      torch.zeros(nz, device="cuda"), n)
    FBPFilter(ne, P, nz, "float32").filter(tmp, w, None)
    ref = tmp[:, :, pad:pad + n]
    f = TCFilter(n, P, nz)
    f.set_kernels(wf, ne, center)
    hi, lo = split16(x)
    out = torch.empty((nz, P, n), device="cuda")
    f.apply(hi, lo, out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu(), ref.cpu()) < 5e-5


@pytest.mark.gpu
def test_tc_filter_per_slice_kernels_and_pairs(cuda):
    """nkern = nz kernels with distinct centre shifts; paired complex output."""
    from tomocupy_b200.reconstruction.tcfilter import TCFilter
    n, P, nz, center = 256, 130, 4, 127.0
    ne = 4 * n
    wf = np_tomo.calc_filter(ne, "parzen")
    rows = _rows(nz, P, n, seed=7)
    shs = np.array([0.0, 0.75, -1.5, 2.25])
    want = np.stack([np_tomo.fbp_filter_center(rows[z:z + 1].astype(np.float64), wf, center,
                                               shs[z], np.float64)[0] for z in range(nz)])
    x = torch.as_tensor(rows, device="cuda")
    hi, lo = split16(x)
    f = TCFilter(n, P, nz, nkern=nz)
    f.set_kernels(wf, ne, center, shs)
    rowsout = torch.empty((nz, P, n), device="cuda")
    f.apply(hi, lo, rowsout)
    pairs = torch.empty((nz // 2, P, n), dtype=torch.complex64, device="cuda")
    f.apply(hi, lo, pairs, pairs=True)
    torch.cuda.synchronize()
    assert rel_l2(rowsout.cpu().double(), torch.as_tensor(want)) < 5e-5
    assert torch.equal(pairs.real.cpu(), rowsout[:nz // 2].cpu())
    assert torch.equal(pairs.imag.cpu(), rowsout[nz // 2:].cpu())
    # a slice range starting at kernel 2 picks kernels 2 and 3
    part = torch.empty((2, P, n), device="cuda")
    f.apply(hi[2:].contiguous(), lo[2:].contiguous(), part, kern0=2)
    torch.cuda.synchronize()
    assert torch.equal(part.cpu(), rowsout[2:].cpu())
    assert not f.timed_out()


@pytest.mark.gpu
def test_prep_split16_matches_fp32_prep(cuda):
    from tomocupy_b200 import synthetic
    from tomocupy_b200.processing.proc_functions import (darkflat_stats, prep_rows,
                                                          prep_rows_split16)
    data, dark, flat, theta, _ = synthetic.make_dataset(90, 4, 128, seed=1)
    data, dark, flat = data.cuda(), dark.cuda(), flat.cuda()
    d0, f0, _ = darkflat_stats(dark, flat)
    P, nz, n = data.shape
    ref = torch.empty((nz, P, n), device="cuda")
    prep_rows(ref, data, d0, f0, out_zstride=P * n, out_pstride=n)
    hi = torch.empty((nz, P, n), dtype=torch.float16, device="cuda")
    lo = torch.empty_like(hi)
    prep_rows_split16(hi, lo, data, d0, f0, out_zstride=P * n, out_pstride=n)
    torch.cuda.synchronize()
    assert torch.equal(hi, ref.half())
    assert torch.equal(lo, (ref - ref.half().float()).half())
