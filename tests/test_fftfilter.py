"""Fused fp32 filter: the circular-convolution statement of the filter chain
(CPU) and the shared-memory FFT kernel against the FP64 oracle, the fp32
cuFFT chain and numpy's FFT for the spectrum output (GPU).

The convolution identity (edge pad -> length-ne circular convolution -> crop
== length-L circular convolution + two folded padding columns) is exact
algebra, checked on the CPU to float64 round-off against the oracle's FP64
fbp_filter_center.  On the GPU the fp32 kernel is held to the accuracy of
the reference's own fp32 chain: its rel-L2 against FP64 must stay within
1.5x that of the oracle's fp32 restatement of the chain (edge pad, fp32
R2C, x complex64 w, C2R, crop) on the same rows.  Both are far above fp32
epsilon on these rows (2e-6 at n = 512, 9e-6 at n = 2048) because the
ramp filter's output is a small difference of large sums: the rows' norm
is 600-1200x the filtered norm.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

from oracle import np_tomo
from tomocupy_b200.reconstruction.fftfilter import operator_columns
from tomocupy_b200.reconstruction.tcfilter import impulse_responses, toeplitz_operator


def _rows(nz, P, n, seed=0):
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, n)
    base = np.clip(1 - x[None, None, :] ** 2, 0, None) * rng.uniform(0.5, 3, (nz, P, 1))
    return (base + 0.01 * rng.standard_normal((nz, P, n))).astype(np.float64)


def _conv(x, hz, n, pad):
    hL, A, B = operator_columns(hz, n, pad)
    L = hL.size
    xL = np.zeros(x.shape[:-1] + (L,))
    xL[..., :n] = x
    y = np.fft.ifft(np.fft.fft(xL) * np.fft.fft(hL)).real[..., :n]
    return y + x[..., :1] * A + x[..., n - 1:n] * B


@pytest.mark.parametrize("name,n,center,sht", [("parzen", 32, 16.0, 0.0),
                                               ("shepp", 200, 90.25, 1.5),
                                               ("ramp", 256, 140.0, -2.375),
                                               ("shepp", 1000, 500.0, 0.5)])
def test_convolution_equals_fp64_filter_chain(name, n, center, sht):
    ne = 4 * n
    wf = np_tomo.calc_filter(ne, name)
    rows = _rows(1, 4, n)
    want = np_tomo.fbp_filter_center(rows, wf, center, sht, np.float64)
    hz = impulse_responses(wf, ne, n, center, sht)[0]
    got = _conv(rows[0], hz, n, ne // 2 - n // 2)
    assert np.abs(got - want[0]).max() <= 1e-10 * np.abs(want).max()
    T = toeplitz_operator(hz, n, ne // 2 - n // 2)
    assert np.abs(got - rows[0] @ T.T).max() <= 1e-10 * np.abs(want).max()


def test_convolution_length_is_power_of_two_at_least_2n():
    for n in (2, 100, 128, 129, 2048, 4096):
        hz = np.arange(4 * n, dtype=np.float64)
        hL, A, B = operator_columns(hz, n, 2 * n - n // 2)
        L = hL.size
        assert L >= 2 * n and L & (L - 1) == 0 and L >= 256
        assert A.shape == (n,) and B.shape == (n,)


@pytest.mark.gpu
@pytest.mark.parametrize("n,P,nz,name,center", [(512, 360, 4, "parzen", 256.0),
                                                (2048, 150, 2, "shepp", 1023.0),
                                                (320, 77, 3, "ramp", 150.5),
                                                (4096, 20, 2, "shepp", 2040.0),
                                                (130, 33, 5, "hann", 60.0)])
def test_fft_filter_rows_vs_fp64_oracle(cuda, n, P, nz, name, center):
    from tomocupy_b200.reconstruction.fftfilter import FFTFilter
    ne = 4 * n
    wf = np_tomo.calc_filter(ne, name)
    rows = _rows(nz, P, n, seed=n)
    want = np_tomo.fbp_filter_center(rows, wf, center, 0.0, np.float64)
    x = torch.as_tensor(rows.astype(np.float32), device="cuda")
    f = FFTFilter(n, P, nz)
    f.set_kernels(wf, ne, center, 0.0)
    out = torch.full((nz, P, n), float("nan"), device="cuda")
    f.apply(x, out, "rows")
    torch.cuda.synchronize()
    err = rel_l2(out.cpu().double(), torch.as_tensor(want))
    ref32 = np_tomo.fbp_filter_center(rows.astype(np.float32), wf, center, 0.0, np.float32)
    err_ref = rel_l2(torch.as_tensor(ref32).double(), torch.as_tensor(want))
    print(f"fft filter n={n}: rel-L2 vs FP64 {err:.2e} (fp32 reference chain {err_ref:.2e})")
    assert err < 1.5 * err_ref + 1e-7, (err, err_ref)
    f.free()


@pytest.mark.gpu
def test_fft_filter_matches_fp32_cufft_filter(cuda):
    """Against the drop-in fp32 chain (edge pad, cuFFT R2C, x w, C2R, crop)."""
    from tomocupy_b200.reconstruction.backproj_functions import phase_weights, rfftfreq32
    from tomocupy_b200.reconstruction.fbp_filter import FBPFilter
    from tomocupy_b200.reconstruction.fftfilter import FFTFilter
    n, P, nz, center = 1024, 200, 4, 511.0
    ne = 4 * n
    pad = ne // 2 - n // 2
    wf = np_tomo.calc_filter(ne, "shepp")
    x = torch.as_tensor(_rows(nz, P, n, seed=3).astype(np.float32), device="cuda")
    tmp = torch.empty((nz, P, ne), device="cuda")
    tmp[:, :, pad:pad + n] = x
    tmp[:, :, :pad] = x[:, :, :1]
    tmp[:, :, pad + n:] = x[:, :, -1:]
    w = phase_weights(torch.as_tensor(wf, device="cuda"), rfftfreq32(ne, "cuda"), center,
                      torch.zeros(nz, device="cuda"), n)
    FBPFilter(ne, P, nz, "float32").filter(tmp, w, None)
    ref = tmp[:, :, pad:pad + n]
    f = FFTFilter(n, P, nz)
    f.set_kernels(wf, ne, center)
    out = torch.empty((nz, P, n), device="cuda")
    f.apply(x, out, "rows")
    torch.cuda.synchronize()
    # two fp32 computations of an ill-conditioned map: compare each with FP64
    want = torch.as_tensor(np_tomo.fbp_filter_center(_rows(nz, P, n, seed=3), wf, center, 0.0,
                                                     np.float64))
    err, err_cufft = rel_l2(out.cpu().double(), want), rel_l2(ref.cpu().double(), want)
    print(f"fft filter vs FP64 {err:.2e}, cuFFT chain vs FP64 {err_cufft:.2e}")
    assert err < 1.5 * err_cufft + 1e-7, (err, err_cufft)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [256, 1024])
def test_fft_filter_per_slice_kernels_pairs_and_spectrum(cuda, n):
    """nkern = nz kernels with distinct centre shifts (two kernels in one complex
    transform); packed complex output; the fused projection FFT; kern0."""
    from tomocupy_b200.reconstruction.fftfilter import FFTFilter
    P, nz, center = 130, 4, n / 2 - 1
    ne = 4 * n
    wf = np_tomo.calc_filter(ne, "parzen")
    rows = _rows(nz, P, n, seed=7)
    shs = np.array([0.0, 0.75, -1.5, 2.25])
    want = np.stack([np_tomo.fbp_filter_center(rows[z:z + 1], wf, center, shs[z],
                                               np.float64)[0] for z in range(nz)])
    ref32 = np.stack([np_tomo.fbp_filter_center(rows[z:z + 1].astype(np.float32), wf, center,
                                                shs[z], np.float32)[0] for z in range(nz)])
    tol = 1.5 * rel_l2(torch.as_tensor(ref32).double(), torch.as_tensor(want)) + 1e-7
    x = torch.as_tensor(rows.astype(np.float32), device="cuda")
    f = FFTFilter(n, P, nz, nkern=nz)
    f.set_kernels(wf, ne, center, shs)
    rowsout = torch.empty((nz, P, n), device="cuda")
    f.apply(x, rowsout, "rows")
    pairs = torch.empty((nz // 2, P, n), dtype=torch.complex64, device="cuda")
    f.apply(x, pairs, "pairs")
    spec = torch.empty_like(pairs)
    f.apply(x, spec, "spectrum")
    torch.cuda.synchronize()
    assert rel_l2(rowsout.cpu().double(), torch.as_tensor(want)) < tol
    assert torch.equal(pairs.real.cpu(), rowsout[:nz // 2].cpu())
    assert torch.equal(pairs.imag.cpu(), rowsout[nz // 2:].cpu())
    packed = want[:nz // 2] + 1j * want[nz // 2:]
    assert rel_l2(spec.cpu().numpy(), np.fft.fft(packed, axis=-1)) < tol
    part = torch.empty((2, P, n), device="cuda")
    f.apply(x[2:].contiguous(), part, "rows", kern0=2)
    torch.cuda.synchronize()
    # slices 2 and 3 of the call pair with each other now (one complex transform)
    assert rel_l2(part.cpu().double(), torch.as_tensor(want[2:])) < 2 * tol


@pytest.mark.gpu
def test_fft_filter_rejects_bad_arguments(cuda):
    from tomocupy_b200 import _lib
    from tomocupy_b200.reconstruction.fftfilter import FFTFilter
    n, P = 200, 10
    f = FFTFilter(n, P, 4)
    wf = np_tomo.calc_filter(4 * n, "shepp")
    x = torch.zeros((4, P, n), device="cuda")
    out = torch.empty((2, P, n), dtype=torch.complex64, device="cuda")
    with pytest.raises(_lib.TcbError):  # set_kernels not called yet
        f.apply(x, out, "pairs")
    f.set_kernels(wf, 4 * n, n / 2)
    with pytest.raises(_lib.TcbError):  # spectrum needs a power-of-two width
        f.apply(x, out, "spectrum")
    with pytest.raises(_lib.TcbError):  # more slices than the handle was made for
        f.apply(torch.zeros((6, P, n), device="cuda"), torch.empty((6, P, n), device="cuda"))
    f.free()
