"""Request server: results in a concurrent mix equal the same requests run
alone, batching and the memory budget behave as documented."""
import threading

import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import serve
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-10


def _alone(req, p, a, b):
    """The same request through the context API, nothing else running."""
    import torch
    ctx = so3.Context(0)
    if req["kind"] == "inverse":
        out = ctx.inverse_batch([a], p, req["precision"])[0]
    elif req["kind"] == "forward":
        out = ctx.forward_batch([a], p, req["precision"])[0]
    else:
        h = ctx.s2toso3(p, a, b)
        out = ctx.inverse(h, p)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_mix_equals_alone():
    import torch
    trace = serve.make_trace(60, rate=2000.0, seed=3, L_range=(8, 96), N_max=12, p_inverse=0.5, p_convolve=0.15)
    for i, r in enumerate(trace):
        r["precision"] = "mixed" if i % 2 else "fp64"
    # a few requests with identical parameters so that split-precision batching occurs
    for i in range(6):
        trace.append({"t": trace[-1]["t"] + 1e-6, "kind": "inverse", "L": 40, "N": 6, "seed": 77 + i,
                      "precision": "mixed"})
    with serve.Server(0, memory_budget=4 << 30, max_inflight=6, max_batch=4, max_L=128) as sv:
        res, wall, outs = serve.replay(sv, trace, keep_outputs=True)
        st = sv.stats()
    assert all(r.status == 0 for r in res)
    assert st["completed"] == len(trace)
    assert any(r.batch > 1 for r in res)  # continuous batching happened
    assert st["peak_bytes"] <= 4 << 30
    for req, out, r in zip(trace, outs, res):
        p, a, b, _ = serve.request_buffers(req)
        ref = _alone(req, p, a, b)
        got = out.cpu().numpy()
        tol = TOL_MIXED if req["precision"] == "mixed" and req["kind"] != "convolve" else TOL_FP64
        assert rel_err(got, ref) <= tol, (req, r)
        if req["precision"] == "fp64" or req["kind"] == "convolve":
            assert np.array_equal(got, ref)  # identical kernels, same arithmetic


def test_submission_from_several_threads():
    import torch
    trace = serve.make_trace(24, rate=1e5, seed=9, L_range=(8, 48), N_max=8)
    bufs = [serve.request_buffers(r) for r in trace]
    torch.cuda.synchronize()
    ids = [None] * len(trace)
    with serve.Server(0, memory_budget=2 << 30, max_inflight=4, max_batch=8, max_L=64) as sv:
        def worker(k):
            for i in range(k, len(trace), 4):
                p, a, b, o = bufs[i]
                ids[i] = sv.submit(trace[i]["kind"], p, a, o, "fp64", inp2=b)
        th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        res = [sv.wait(i) for i in ids]
    assert all(r.status == 0 for r in res)
    for req, (p, a, b, o) in zip(trace, bufs):
        assert np.array_equal(o.cpu().numpy(), _alone(req, p, a, b))


def test_budget_rejects_oversized_request_and_serves_the_rest():
    import torch
    small = {"t": 0.0, "kind": "inverse", "L": 16, "N": 4, "seed": 1, "precision": "fp64"}
    big = {"t": 0.0, "kind": "inverse", "L": 128, "N": 32, "seed": 2, "precision": "fp64"}
    # 24 MiB: the resident Delta tables to L=128 (11.3 MB for both recursions) plus room for
    # the small request's scratch and buffers, not for the big one's (about 70 MB)
    with serve.Server(0, memory_budget=24 << 20, max_inflight=2, max_batch=1, max_L=128) as sv:
        pb, ab, _, ob = serve.request_buffers(big)
        ps, as_, _, os_ = serve.request_buffers(small)
        torch.cuda.synchronize()
        i_big = sv.submit("inverse", pb, ab, ob)
        i_small = sv.submit("inverse", ps, as_, os_)
        r_big, r_small = sv.wait(i_big), sv.wait(i_small)
    assert r_big.status == 4
    assert r_small.status == 0
    assert np.array_equal(os_.cpu().numpy(), _alone(small, ps, as_, None))


def test_latency_fields():
    trace = serve.make_trace(20, rate=500.0, seed=5, L_range=(8, 32), N_max=4)
    with serve.Server(0, memory_budget=1 << 30, max_inflight=4, max_L=32) as sv:
        res, wall, _ = serve.replay(sv, trace)
    s = serve.latency_summary(res, wall)
    assert s["requests"] == 20 and s["failed"] == 0
    assert 0 < s["p50_ms"] <= s["p99_ms"]
    assert all(0 <= r.queue_us <= r.total_us for r in res)


def test_split_requests_of_different_geometries_batch():
    """Split-precision requests of different (L, N) form ragged units (one
    tensor-core launch); each result matches its FP64 transform."""
    import torch
    trace = serve.make_trace(40, rate=1e5, seed=21, L_range=(24, 40), N_max=6, p_inverse=1.0, precision="mixed")
    with serve.Server(0, memory_budget=8 << 30, max_inflight=2, max_batch=16, max_L=64) as sv:
        res, wall, outs = serve.replay(sv, trace, keep_outputs=True)
    assert all(r.status == 0 for r in res)
    assert max(r.batch for r in res) >= 4
    ctx = so3.Context(0)
    for req, out in zip(trace, outs):
        p, a, b, _ = serve.request_buffers(req)
        ref = ctx.inverse(a, p)
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) <= TOL_MIXED
