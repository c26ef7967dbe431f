"""Serving loop: continuous batching of uneven requests (tomocupy_b200.serving).

The per-request computation is the fused reconstruction of GPURec; here the
tests check what the serving layer adds: results identical alone and in a
mix (bit for bit when every chunk holds one request; within 1e-6 when
chunks pack several requests of one geometry), agreement with GPURec,
admission under an HBM budget, and the request generator.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from tomocupy_b200.serving import latency_summary, poisson_stream


def test_poisson_stream_is_seeded_and_balanced():
    a = poisson_stream(rate=50, count=40, seed=3)
    b = poisson_stream(rate=50, count=40, seed=3)
    assert a == b
    t = np.array([x[0] for x in a])
    assert np.all(np.diff(t) > 0)
    assert {x[4] for x in a} == {"float32", "mixed"}
    assert sum(x[4] == "mixed" for x in a) == 20
    assert all(1 <= x[3] <= 64 for x in a)


def test_latency_summary():
    class R:
        def __init__(self, a, d, w):
            self.arrival, self.t_done, self.gups_work = a, d, w
            self.latency = d - a
    rs = [R(0.0, 0.010, 1e9), R(0.005, 0.025, 1e9)]
    s = latency_summary(rs)
    assert abs(s["p50_ms"] - 15.0) < 1e-9 and s["requests"] == 2
    assert abs(s["GUPS"] - 2e9 / 0.025 / 1e9) < 1e-9


def _requests(specs, seed=0):
    from tomocupy_b200 import synthetic
    from tomocupy_b200.serving import Request
    out = []
    for k, (n, P, nz, prec) in enumerate(specs):
        data, dark, flat, theta, _ = synthetic.make_dataset(P, nz, n, seed=seed + k)
        out.append(Request(k, data.pin_memory(), dark.pin_memory(), flat.pin_memory(), theta,
                           n / 2, prec, "parzen", arrival=0.002 * k))
    return out


SPECS = [(128, 90, 3, "float32"), (256, 180, 9, "mixed"), (128, 90, 16, "mixed"),
         (256, 120, 5, "float32"), (128, 90, 7, "float32")]


@pytest.mark.gpu
def test_results_identical_alone_and_in_mix(cuda):
    """Without packing every chunk holds one request's slices: bit for bit."""
    from tomocupy_b200.serving import Server
    mix = _requests(SPECS)
    srv = Server(ncz=8, pack=False)
    srv.serve(mix, realtime=False)
    assert srv.peak_active >= 2  # they really overlapped
    for r in mix:
        alone = _requests([SPECS[r.rid]], seed=r.rid)[0]
        alone.rid = r.rid
        Server(ncz=8, pack=False).serve([alone], realtime=False)
        assert torch.equal(alone.out, r.out), r.rid
        assert np.isfinite(r.latency) and r.t_done >= r.t_admit


@pytest.mark.gpu
def test_packed_chunks_match_alone(cuda):
    """Mixed-precision requests of one geometry share chunk launches (3 + 5
    slices of 128 x 90 fill one chunk of 8, the 4 of the third one the
    next); a slice may then be paired with another request's slice in
    fourierrec's real/imaginary packing, whose crosstalk (the reference's
    too) stays within the mixed-precision budget.  fp32 requests of one
    geometry are not packed."""
    from tomocupy_b200.serving import Server
    specs = [(128, 90, 3, "mixed"), (256, 180, 9, "mixed"), (128, 90, 5, "mixed"),
             (128, 90, 4, "mixed")]
    mix = _requests(specs)
    srv = Server(ncz=8, pack=True)
    srv.serve(mix, realtime=False)
    unpacked = Server(ncz=8, pack=False)
    unpacked.serve(_requests(specs), realtime=False)
    assert (srv.chunks, unpacked.chunks) == (4, 5), (srv.chunks, unpacked.chunks)
    for r in mix:
        alone = _requests([specs[r.rid]], seed=r.rid)[0]
        Server(ncz=8).serve([alone], realtime=False)
        err = rel_l2(r.out, alone.out)
        print(f"request {r.rid}: packed vs alone {err:.2e}")
        assert err < 1e-3, (r.rid, err)
    fp32 = [(128, 90, 3, "float32"), (128, 90, 5, "float32")]
    srv32 = Server(ncz=8, pack=True)
    srv32.serve(_requests(fp32), realtime=False)
    assert srv32.chunks == 2


@pytest.mark.gpu
def test_request_matches_gpurec(cuda):
    from tomocupy_b200 import global_vars
    from tomocupy_b200.dataio import ArrayReader, ArrayWriter
    from tomocupy_b200.rec import GPURec
    from tomocupy_b200.serving import Server
    req = _requests([(256, 180, 16, "float32")], seed=11)[0]
    Server(ncz=8).serve([req], realtime=False)
    global_vars.reset(reconstruction_algorithm="fourierrec", nsino_per_chunk=8)
    writer = ArrayWriter(device="cpu", pin=True)
    GPURec(ArrayReader(req.frames, req.dark, req.flat, theta=req.theta, pin=True),
           writer).recon_all()
    # the server grids with the fp32 register kernel (no per-geometry weight
    # tables), GPURec on the tensor cores with streamed weights: the two agree
    # within the fourierrec tolerance
    assert rel_l2(req.out, writer.rec) < 1e-5


@pytest.mark.gpu
def test_admission_holds_the_budget(cuda):
    from tomocupy_b200.serving import Server
    reqs = _requests([(128, 90, 8, "float32")] * 4)
    srv = Server(ncz=8)
    srv.warm(reqs[:1])
    one = srv._request_bytes(reqs[0])
    # room for the resident geometry and one request only
    srv.budget = srv.geom_bytes + one + one // 2
    srv.serve(reqs, realtime=False)
    assert srv.peak_active == 1
    assert srv.peak_bytes <= srv.budget
    assert all(np.isfinite(r.t_done) for r in reqs)
