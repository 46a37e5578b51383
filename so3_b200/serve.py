"""Request serving on one GPU: Python face of the so3gpu_server C API.

The loop itself is native (so3_b200/csrc/server.cpp): continuous batching of
split-precision requests with identical parameters, one CUDA stream per
in-flight unit, admission by a device-memory budget, per-request queueing and
total latency.  This module adds device buffers for requests, a seeded
Poisson request trace, and a trace replayer reporting p50 / p99 latency and
throughput.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .api import SO3Parameters, f_size, flmn_size

KINDS = {"inverse": 0, "forward": 1, "convolve": 2}
PRECISIONS = {"fp64": 0, "mixed": 1}


@dataclass
class Done:
    id: int
    queue_us: float
    total_us: float
    batch: int
    status: int


class Server:
    """so3gpu_server bound to one device.  Buffers are torch CUDA tensors that
    the caller keeps alive until the request is done."""

    def __init__(self, device: int = 0, memory_budget: int = 120 << 30, max_inflight: int = 8, max_batch: int = 8,
                 max_L: int = 0):
        self._lib = _lib.load()
        self._s = self._lib.so3gpu_server_create(device, memory_budget, max_inflight, max_batch, max_L)
        if not self._s:
            _lib.check("so3gpu_server_create")
        self.device = device

    def close(self):
        if getattr(self, "_s", None):
            self._lib.so3gpu_server_destroy(self._s)
            self._s = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, kind: str, p: SO3Parameters, inp, out, precision: str = "fp64", inp2=None) -> int:
        q = p.to_struct()
        rid = self._lib.so3gpu_server_submit(self._s, KINDS[kind], ctypes.byref(q), inp.data_ptr(),
                                             inp2.data_ptr() if inp2 is not None else None, out.data_ptr(),
                                             PRECISIONS[precision])
        if rid < 0:
            _lib.check("so3gpu_server_submit")
        return rid

    def _query(self, fn, rid):
        qu, tu = ctypes.c_double(), ctypes.c_double()
        b, st = ctypes.c_int(), ctypes.c_int()
        r = fn(self._s, rid, ctypes.byref(qu), ctypes.byref(tu), ctypes.byref(b), ctypes.byref(st))
        if r < 0:
            raise KeyError(rid)
        return Done(rid, qu.value, tu.value, b.value, st.value) if r == 1 else None

    def wait(self, rid: int) -> Done:
        return self._query(self._lib.so3gpu_server_wait, rid)

    def poll(self, rid: int):
        return self._query(self._lib.so3gpu_server_poll, rid)

    def drain(self):
        self._lib.so3gpu_server_drain(self._s)

    def stats(self) -> dict:
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        d = ctypes.c_size_t()
        self._lib.so3gpu_server_stats(self._s, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
        return {"submitted": a.value, "completed": b.value, "units": c.value, "peak_bytes": d.value}


# --------------------------------------------------------------------- traces
def make_trace(n: int, rate: float, seed: int, L_range=(16, 1024), N_max: int = 64, p_inverse: float = 0.6,
               p_convolve: float = 0.0, precision: str = "fp64", shapes=None):
    """Seeded request trace: Poisson arrivals at `rate` per second; inverse
    with probability p_inverse, directional convolution with p_convolve, else
    forward; complex MW, L log-uniform in L_range (rounded), N uniform in
    [1, min(L, N_max)] -- or, when `shapes` lists (L, N) pairs, one of those
    uniformly (recurring geometries, which split-precision requests batch)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    lo, hi = math.log(L_range[0]), math.log(L_range[1])
    out = []
    for i in range(n):
        if shapes:
            L, N = shapes[int(rng.integers(len(shapes)))]
        else:
            L = int(round(math.exp(rng.uniform(lo, hi))))
            N = int(rng.integers(1, min(L, N_max) + 1))
        u = rng.uniform()
        kind = "inverse" if u < p_inverse else ("convolve" if u < p_inverse + p_convolve else "forward")
        out.append({"t": float(t[i]), "kind": kind, "L": L, "N": N, "seed": int(rng.integers(1 << 31)),
                    "precision": precision})
    return out


def request_buffers(req, device="cuda"):
    """Seeded device input (U(-1,1) real and imaginary parts) and an output
    buffer for one trace request."""
    import torch
    p = SO3Parameters(L=req["L"], N=req["N"])
    g = torch.Generator(device=device)
    g.manual_seed(req["seed"])

    def u(n):
        x = torch.rand(2 * n, dtype=torch.float64, device=device, generator=g) * 2 - 1
        return torch.view_as_complex(x.view(n, 2))

    if req["kind"] == "inverse":
        return p, u(flmn_size(p)), None, torch.empty(f_size(p), dtype=torch.complex128, device=device)
    if req["kind"] == "forward":
        return p, u(f_size(p)), None, torch.zeros(flmn_size(p), dtype=torch.complex128, device=device)
    # directional convolution: flm over all l < L, glm only |m| < min(8, N)
    flm = u(p.L * p.L)
    glm = u(p.L * p.L)
    el = torch.arange(p.L * p.L, device=device)
    l = torch.floor(torch.sqrt(el.double())).long()
    m = el - l * l - l
    glm[m.abs() >= min(8, p.N)] = 0
    return p, flm, glm, torch.empty(f_size(p), dtype=torch.complex128, device=device)


def replay(server: Server, trace, keep_outputs: bool = False, time_scale: float = 1.0):
    """Submits every request at its arrival time (scaled), waits for all, and
    returns (per-request results, wall seconds).  Inputs are generated before
    the clock starts."""
    import torch
    bufs = [request_buffers(r) for r in trace]
    torch.cuda.synchronize()
    ids = []
    t0 = time.perf_counter()
    for r, (p, a, b, o) in zip(trace, bufs):
        dt = r["t"] * time_scale - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        ids.append(server.submit(r["kind"], p, a, o, r["precision"], inp2=b))
    res = [server.wait(i) for i in ids]
    wall = time.perf_counter() - t0
    outs = [b[3] for b in bufs] if keep_outputs else None
    return res, wall, outs


def latency_summary(res, wall):
    tot = sorted(r.total_us for r in res)
    q = sorted(r.queue_us for r in res)

    def pct(v, f):
        return v[min(len(v) - 1, max(0, math.ceil(f * len(v)) - 1))] / 1e3 if v else None

    return {"requests": len(res), "wall_s": wall, "throughput_rps": len(res) / wall if wall > 0 else None,
            "p50_ms": pct(tot, 0.50), "p99_ms": pct(tot, 0.99), "queue_p50_ms": pct(q, 0.50),
            "queue_p99_ms": pct(q, 0.99), "failed": sum(1 for r in res if r.status != 0),
            "mean_batch": float(np.mean([r.batch for r in res])) if res else None}


def replay_stream(server: Server, trace, time_scale: float = 1.0, seed: int = 5, timeout_s: float = 600.0,
                  max_out_bytes: int = 16 << 30):
    """Replays a trace of arbitrary length with bounded device memory.  The
    inverse and forward inputs of every request are prefixes of one seeded
    pool of U(-1,1) complex values as large as the largest input of the trace
    (transforms read no entry outside their band limits, so any prefix is a
    valid input); directional-convolution requests get their own buffers.
    Every request gets its own output buffer at submission, released once it
    has completed; while the outstanding outputs exceed max_out_bytes the
    client waits for its oldest request before submitting the next (a client
    with bounded memory: at offered rates above capacity the submissions
    then follow the completions).  Returns (results, wall seconds); raises TimeoutError when
    requests are still pending timeout_s after the first submission."""
    import torch
    need = 0
    for r in trace:
        if r["kind"] != "convolve":
            p = SO3Parameters(L=r["L"], N=r["N"])
            need = max(need, flmn_size(p) if r["kind"] == "inverse" else f_size(p))
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    pool = torch.view_as_complex((torch.rand(2 * max(need, 1), dtype=torch.float64, device="cuda", generator=g) * 2
                                  - 1).view(-1, 2))
    conv = {}
    torch.cuda.synchronize()
    live, done = {}, {}
    live_bytes = 0
    ids = []
    t0 = time.perf_counter()
    for r in trace:
        dt = r["t"] * time_scale - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        p = SO3Parameters(L=r["L"], N=r["N"])
        b = None
        if r["kind"] == "inverse":
            a, n_out = pool[:flmn_size(p)], f_size(p)
        elif r["kind"] == "forward":
            a, n_out = pool[:f_size(p)], flmn_size(p)
        else:
            key = (r["L"], r["N"])
            if key not in conv:
                conv[key] = request_buffers(r)[1:3]
            (a, b), n_out = conv[key], f_size(p)
        while live and live_bytes + 16 * n_out > max_out_bytes:  # bounded client memory
            k = next(iter(live))
            done[k] = server.wait(k)
            live_bytes -= live.pop(k).numel() * 16
        out = torch.empty(n_out, dtype=torch.complex128, device="cuda")
        rid = server.submit(r["kind"], p, a, out, r["precision"], inp2=b)
        ids.append(rid)
        live[rid] = out
        live_bytes += 16 * n_out
        for k in list(live):  # a completed poll hands over (and forgets) the record
            d = server.poll(k)
            if d is not None:
                done[k] = d
                live_bytes -= live.pop(k).numel() * 16
    while live:  # bounded: a request that never completes raises instead of blocking forever
        for k in list(live):
            d = server.poll(k)
            if d is not None:
                done[k] = d
                del live[k]
        if live:
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError(f"{len(live)} requests still pending after {timeout_s:g} s")
            time.sleep(0.001)
    wall = time.perf_counter() - t0
    live.clear()
    return [done[i] for i in ids], wall


def serving_run(n: int = 400, rate: float = 200.0, seed: int = 11, precision: str = "fp64",
                budget: int = 120 << 30, max_inflight: int = 8, max_batch: int = 8, device: int = 0,
                L_range=(16, 1024), N_max: int = 64, shapes=None):
    """The serving trace workload (inverse 60 % / forward 40 %, complex MW,
    L log-uniform, N uniform in [1, min(L, N_max)] or drawn from `shapes`,
    U(-1,1) inputs, Poisson arrivals at `rate`) through a Server: latency
    percentiles and throughput."""
    trace = make_trace(n, rate, seed, L_range=L_range, N_max=N_max, p_inverse=0.6, precision=precision,
                       shapes=shapes)
    max_L = max(L for L, _ in shapes) if shapes else L_range[1]
    with Server(device, memory_budget=budget, max_inflight=max_inflight, max_batch=max_batch,
                max_L=max_L) as sv:
        res, wall = replay_stream(sv, trace)
        st = sv.stats()
    out = latency_summary(res, wall)
    out.update({"offered_rate_rps": rate, "precision": precision, "peak_scratch_bytes": st["peak_bytes"],
                "units": st["units"]})
    return out
