"""tcb_prep_noalloc: frame normalisation for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc where they normalise frames (an
acquisition loop that must not allocate once streaming has started, or code
running inside a runtime that owns the device allocator).  For them the
library keeps the dark/flat statistics in a fixed device array of its own.
This file checks, through the C ABI, that two calls in a row give exactly
what the allocating entry points give (tcb_darkflat_stats + tcb_prep_rows,
whose statistics live in buffers the caller allocates), and that a size over
the fixed maximum is refused before any GPU work.  It is named so that
pytest collects it last.
"""
import pytest
import torch

from tomocupy_b200 import _lib


_CODES = {torch.uint16: _lib.TCB_U16, torch.uint8: _lib.TCB_U8, torch.float32: _lib.TCB_F32}


def _noalloc(out, data, dark, flat, flags, xoff=0, width=None):
    nproj, nz, n = data.shape
    _lib.call("tcb_prep_noalloc", out.data_ptr(), data.data_ptr(), dark.data_ptr(),
              flat.data_ptr(), nproj, nz, n, dark.shape[0], flat.shape[0],
              _CODES[data.dtype], 1.0, nproj * out.shape[-1], out.shape[-1], 0, xoff,
              width if width is not None else xoff + n, flags,
              torch.cuda.current_stream().cuda_stream)


def _allocating(out, data, dark, flat, flags, xoff=0, width=None):
    nproj, nz, n = data.shape
    dev = data.device
    dark0 = torch.empty((nz, n), dtype=torch.float32, device=dev)
    flat0 = torch.empty((nz, n), dtype=torch.float32, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    _lib.call("tcb_darkflat_stats", dark0.data_ptr(), flat0.data_ptr(), 0, dark.data_ptr(),
              flat.data_ptr(), dark.shape[0], flat.shape[0], nz, n, _CODES[data.dtype], 1.0, 0,
              s)
    _lib.call("tcb_prep_rows", out.data_ptr(), data.data_ptr(), dark0.data_ptr(),
              flat0.data_ptr(), 0, nproj, nz, n, nz * n, n, _CODES[data.dtype],
              nproj * out.shape[-1], out.shape[-1], 0, xoff,
              width if width is not None else xoff + n, flags | _lib.PREP_DARKFLAT, s)


@pytest.mark.gpu
def test_noalloc_matches_allocating_path_twice():
    from tomocupy_b200 import synthetic
    assert torch.cuda.is_available()
    dev = torch.device("cuda")
    cases = [
        # (nproj, nz, n, seed, flags, xoff, width, dtype): plain -log, edge-padded
        # rows, 8-bit and float32 frames, and the largest plane the fixed
        # statistics hold (nz * n = TCB_NOALLOC_MAX_PLANE: both halves of the
        # array used to the end)
        (90, 6, 200, 21, _lib.PREP_MINUS_LOG, 0, None, torch.uint16),
        (60, 8, 256, 22, _lib.PREP_MINUS_LOG | _lib.PREP_EDGE_PAD, 384, 1024, torch.uint16),
        (40, 4, 128, 23, _lib.PREP_MINUS_LOG, 0, None, torch.uint8),
        (40, 4, 128, 24, _lib.PREP_MINUS_LOG, 0, None, torch.float32),
        (3, 512, 2048, 25, _lib.PREP_MINUS_LOG, 0, None, torch.uint16),
    ]
    for nproj, nz, n, seed, flags, xoff, width, dt in cases:
        data, dark, flat, _, _ = synthetic.make_dataset(nproj, nz, n, seed=seed)
        if dt == torch.uint8:   # 8-bit frames: counts scaled into [0, 255]
            data, dark, flat = ((t.to(torch.int32) // 64).clamp(0, 255).to(torch.uint8)
                                for t in (data, dark, flat))
        elif dt == torch.float32:
            data, dark, flat = (t.to(torch.float32) for t in (data, dark, flat))
        data, dark, flat = data.to(dev), dark.to(dev), flat.to(dev)
        w = width if width is not None else n
        got = torch.full((nz, nproj, w), float("nan"), device=dev)
        want = torch.full((nz, nproj, w), float("nan"), device=dev)
        _noalloc(got, data, dark, flat, flags, xoff, width)
        _allocating(want, data, dark, flat, flags, xoff, width)
        torch.cuda.synchronize()
        # same kernels and operation order: bit-identical (the prep tolerance)
        assert torch.equal(got, want), (nproj, nz, n)


def test_noalloc_rejects_oversized_chunk_without_gpu_work():
    """nz*n above the fixed maximum is an argument error raised on the host."""
    big_nz, n = 1024, 2048  # 2M elements > TCB_NOALLOC_MAX_PLANE (1M)
    with pytest.raises(_lib.TcbError) as e:
        _lib.call("tcb_prep_noalloc", 16, 16, 16, 16, 10, big_nz, n, 10, 10, _lib.TCB_U16, 1.0,
                  10 * n, n, 0, 0, n, _lib.PREP_MINUS_LOG, 0)
    assert e.value.status == 1
    assert "exceeds the fixed scratch" in str(e.value)
