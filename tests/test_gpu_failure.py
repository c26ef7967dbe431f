"""Failure detection of the bounded waits, without a GPU fault.

The tensor-core filter, the tensor-core gridding and the TMA-staged line
backprojection wait on mbarriers with a clock budget; when it runs out the
kernel records the expiry and finishes instead of hanging.
tcb_check_bounded_wait runs that same wait on an mbarrier that nothing
arrives on (nothing in flight, no TMEM held), with a budget of about a
millisecond, so the wait must run out.  The test checks that the expiry is
reported, that the call returns, and that the context still runs a
reconstruction afterwards."""
import ctypes as C

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_bounded_wait_expires_and_context_survives(cuda):
    from tomocupy_b200 import _lib, cfunc_fourierrec
    budget = 2_000_000  # SM cycles, ~1 ms at 1.9 GHz
    timed_out, waited = C.c_int(0), C.c_longlong(0)
    _lib.call("tcb_check_bounded_wait", budget, C.byref(timed_out), C.byref(waited),
              _lib.stream_ptr(None))
    assert timed_out.value == 1
    assert budget < waited.value < 100 * budget
    # the context is intact: a tensor-core gridding run (which uses the same
    # waits) completes without reporting an expiry
    n, nproj, nz = 128, 90, 2
    theta = torch.arange(nproj, dtype=torch.float32, device=cuda) * (3.14159265 / nproj)
    op = cfunc_fourierrec.cfunc_fourierrec(nproj, nz, n, theta)
    op.set_gridding(_lib.GRID_TENSOR)
    f = torch.empty((nz, n, n, 2), device=cuda)
    op.backprojection(f, torch.randn((nz, nproj, n, 2), device=cuda), None)
    torch.cuda.synchronize()
    assert not op.timed_out()
    assert torch.isfinite(f).all()
    op.free()
