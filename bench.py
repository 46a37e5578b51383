#!/usr/bin/env python
"""Benchmark of the SO(3) Wigner transform path on B200.

One step = one complex inverse transform plus one forward transform
(so3_core_inverse_via_ssht then so3_core_forward_via_ssht semantics) of one
signal at L=512, N=64, MW sampling, L0=0, padded storage, negative-first
n-order, all n, Risbo recursion, with flmn real and imaginary parts iid
U(-1, 1) (seeded, per rank).  The metric is transforms per second (one
inverse + one forward = one transform unit); ranks run independent signals
(weak scaling, no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "inv+fwd transforms/s at L=512,N=64: mixed vs FP64 GPU at ≤1e-10 rel err; p99"
UNIT = "transforms/s"


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--L", type=int, default=512)
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def workload(L, N):
    return {"workload": f"complex MW inverse+forward, L={L}, N={N}, L0=0, padded, negative-first, "
                        f"n_mode=ALL, Risbo, flmn U(-1,1) seeded per rank",
            "L": L, "N": N, "sampling": "MW", "storage": "padded", "dl_method": "Risbo",
            "l2": "inputs larger than L2 (flmn %.0f MB, f %.0f MB per signal)" % (
                (2 * N - 1) * L * L * 16 / 1e6, (2 * N - 1) * L * (2 * L - 1) * 16 / 1e6),
            "parallelism": "independent signals per rank (replicas)"}


def contraction_macs(L, N):
    """Algorithmic complex-by-real multiply-adds of one Wigner contraction
    (one direction), m' >= 0 fold: sum_n sum_{l>=|n|} (l+1)(2l+1)."""
    tot = 0
    for n in range(-(N - 1), N):
        for l in range(abs(n), L):
            tot += (l + 1) * (2 * l + 1)
    return tot


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.file.name).read().strip().splitlines()]
            os.unlink(self.file.name)
        except Exception:
            return None
        rows = [[x.strip() for x in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------- CPU side
def _cpu_sample_worker(args):
    """One bounded sample of the reference's own CPU path (run in a spawned
    process): so3_core_inverse_via_ssht + so3_core_forward_via_ssht at the
    bench's L and N restricted to n_mode=MAXIMUM (2 of the 2N-1 n-planes per
    direction), plus the gamma-axis FFT passes alone, so the full unit can be
    rebuilt as t_gamma + (2N-1)/2 * (t_sample - t_gamma)."""
    L, N, use_ref = args
    import ctypes

    import numpy as np
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from so3_b200 import synth
    p = O.params(L, N, mode=O.MAXIMUM)
    fl = synth.gen_flmn(p, 77, "uniform")
    R = O.ref() if use_ref else None
    f = np.zeros(O.f_size(p), np.complex128)
    out = np.zeros(fl.size, np.complex128)
    t0 = time.perf_counter()
    if R is not None:
        R.so3_core_inverse_via_ssht(f.ctypes.data_as(ctypes.c_void_p), fl.ctypes.data_as(ctypes.c_void_p),
                                    ctypes.byref(p))
        R.so3_core_forward_via_ssht(out.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p),
                                    ctypes.byref(p))
    else:
        f = O.inverse(fl, p)
        O.forward(f, p, out=out)
    t1 = time.perf_counter()
    # the gamma passes (one backward, one forward over all samples)
    stride = L * (2 * L - 1)
    g = np.zeros((2 * N - 1) * stride, np.complex128)
    t2 = time.perf_counter()
    O.dft_strided(g, 2 * N - 1, stride, stride, 1, +1)
    O.dft_strided(g, 2 * N - 1, stride, stride, 1, -1)
    t3 = time.perf_counter()
    return t1 - t0, t3 - t2


def cpu_unit_seconds(L, N, procs):
    """Per-process wall seconds of one full unit, estimated from the sample."""
    import multiprocessing as mp
    from oracle import oracle as O
    O.build()
    use_ref = O.ref() is not None
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_sample_worker, [(L, N, use_ref)] * procs)
    units = []
    for ts, tg in res:
        units.append(tg + (2 * N - 1) / 2.0 * max(ts - tg, 0.0))
    return statistics.median(units), statistics.median([r[0] for r in res]), use_ref


def cpu_procs(L, N):
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 64 << 30
    per = 6.0 * (2 * N - 1) * L * (2 * L - 1) * 16  # a few copies of f per process
    return max(1, min(os.cpu_count() or 1, 32, int(avail * 0.6 // per)))


# --------------------------------------------------------------------- reference arm
def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    procs = cpu_procs(a.L, a.N)
    kind = "reference" if O.ref() is not None else "port"
    for _ in range(a.warmup):
        cpu_unit_seconds(a.L, a.N, procs)
    vals = []
    t0 = time.perf_counter()
    for _ in range(a.steps):
        unit_s, samp_s, _ = cpu_unit_seconds(a.L, a.N, procs)
        vals.append(procs / unit_s)
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    sample = (f"so3_core_inverse_via_ssht + so3_core_forward_via_ssht at L={a.L}, N={a.N}, n_mode=MAXIMUM "
              f"(2 of {2 * a.N - 1} n-planes per direction) per process plus the gamma FFT passes alone, "
              f"scaled to all {2 * a.N - 1} planes; {procs} concurrent processes")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * wall / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload(a.L, a.N),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": kind, "sample": sample,
                             "label": "reference C (so3_core.c, so3_sampling.c, so3_conv.c) + project "
                                      "SSHT/FFTW stand-ins" if kind == "reference" else "oracle port"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- our arm
def run_ours(a):
    import torch
    import torch.distributed as dist

    import so3_b200 as so3
    from so3_b200 import dist as sdist
    from so3_b200 import synth

    info = sdist.rank_info()
    world, rank, local = info.world, info.rank, info.local
    torch.cuda.set_device(local)
    sdist.init("nccl" if world > 1 else None, timeout_s=120)

    L, N = a.L, a.N
    p = so3.SO3Parameters(L=L, N=N, L0=0, sampling_scheme=0, n_order=1, storage=0, n_mode=0, dl_method=0)
    fl_host = synth.gen_flmn(p, sdist.signal_seed(1000, rank, 0), "uniform")
    stream = torch.cuda.current_stream()
    d_flmn = torch.from_numpy(fl_host).to(f"cuda:{local}")
    d_f = torch.empty(so3.f_size(p), dtype=torch.complex128, device=f"cuda:{local}")
    d_back = torch.empty(so3.flmn_size(p), dtype=torch.complex128, device=f"cuda:{local}")
    ctx = so3.Context(local, stream=stream)
    ctx.prepare(p)
    fp64_peak = so3.measure_fp64_peak(local)

    def step():
        ctx.inverse(d_flmn, p, out=d_f)
        ctx.forward(d_f, p, out=d_back)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        sdist.barrier()
    ctx.stage_timing(True)
    ctx.stage_times()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    launches0 = so3.launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        evs[0].record(stream)
        for i in range(a.steps):
            step()
            evs[i + 1].record(stream)
        torch.cuda.synchronize()
    launches = so3.launch_count() - launches0
    stages = ctx.stage_times()
    ctx.stage_timing(False)
    total_ms = evs[0].elapsed_time(evs[-1])
    lat = [evs[i].elapsed_time(evs[i + 1]) for i in range(a.steps)]
    total_ms = sdist.max_over_ranks(total_ms, device=f"cuda:{local}")
    value = sdist.job_throughput(world * a.steps, total_ms / 1e3)
    rt_err = float(((d_back - d_flmn).abs().max() / d_flmn.abs().max()).item())

    # ---- roofline of the dominant kernel
    per = {k: v[0] / v[1] for k, v in stages.items()}
    dom = max(per, key=per.get)
    macs = contraction_macs(L, N)
    f_bytes = (2 * N - 1) * L * (2 * L - 1) * 16
    if "contract" in dom:
        achieved = 4.0 * macs / (per[dom] / 1e3) / 1e12
        roof = {"kernel": dom, "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak,
                "peak_source": "FP64 FMA-chain microbenchmark on this GPU (so3gpu_measure_fp64_peak); the "
                               "measured-peaks file has no FP64 figure",
                "algorithmic": f"4 flops x {macs:.4g} complex-by-real MACs per launch"}
    else:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"] \
            if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
        achieved = 2.0 * f_bytes / (per[dom] / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "algorithmic": f"read+write of the sample array, 2 x {f_bytes} B"}
    roof["traffic"] = traffic_from_profiles(dom, L, N)
    roof["avg_ms"] = per[dom]

    # ---- end to end through the drop-in C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(so3, p, fl_host, a.steps, local, world, dist)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            procs = cpu_procs(L, N)
            unit_s, samp_s, use_ref = cpu_unit_seconds(L, N, procs)
            cpu = {"value": procs / unit_s, "unit": UNIT, "cores": procs,
                   "kind": "reference" if use_ref else "port",
                   "sample": f"inverse+forward at L={L}, N={N} restricted to n_mode=MAXIMUM (2 of {2 * N - 1} "
                             f"n-planes per direction, {samp_s:.1f} s) plus the gamma FFT passes, scaled to all "
                             f"planes; {procs} concurrent single-threaded processes",
                   "seconds_per_unit_per_process": unit_s}
        except Exception as ex:  # the CPU baseline never blocks the GPU line
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload(L, N),
                "precision": "plain FP64 path (the split-precision path is not part of this line)",
                "roundtrip_rel_err": rt_err,
                "latency_ms": {"p50": statistics.median(lat), "p99": sorted(lat)[min(len(lat) - 1,
                                                                                 math.ceil(0.99 * len(lat)) - 1)]},
                "stage_ms": {k: round(v, 4) for k, v in per.items()},
                "gpu_launches": int(launches), "roofline": roof, "e2e": e2e, "cpu_baseline": cpu,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    sdist.finalize()


def run_e2e(so3, p, fl_host, steps, local, world, dist):
    """Same metric through so3_core_{inverse,forward}_via_ssht on pinned host
    buffers: every step copies flmn and f host->device and f and flmn back."""
    import ctypes

    import numpy as np
    import torch

    from so3_b200 import dist as sdist
    lib = so3._lib.load()
    q = p.to_struct()
    fl_pin = torch.from_numpy(fl_host).pin_memory()
    f_pin = torch.empty(so3.f_size(p), dtype=torch.complex128).pin_memory()
    back_pin = torch.empty(so3.flmn_size(p), dtype=torch.complex128).pin_memory()

    def step():
        lib.so3_core_inverse_via_ssht(ctypes.c_void_p(f_pin.data_ptr()), ctypes.c_void_p(fl_pin.data_ptr()),
                                      ctypes.byref(q))
        lib.so3_core_forward_via_ssht(ctypes.c_void_p(back_pin.data_ptr()), ctypes.c_void_p(f_pin.data_ptr()),
                                      ctypes.byref(q))
        so3._lib.check("e2e")

    step()  # warm-up (staging buffers)
    torch.cuda.synchronize()
    if world > 1:
        sdist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    el = time.perf_counter() - t0
    el = sdist.max_over_ranks(el, device=f"cuda:{local}")
    err = float(np.abs(back_pin.numpy() - fl_host).max() / np.abs(fl_host).max())
    nb_fl = fl_host.size * 16
    nb_f = so3.f_size(p) * 16
    return {"value": world * steps / el, "unit": UNIT, "h2d_bytes_per_step": nb_fl + nb_f,
            "d2h_bytes_per_step": nb_f + nb_fl, "api": "so3_core_inverse_via_ssht + so3_core_forward_via_ssht "
                                                       "(host pointers, pinned)", "roundtrip_rel_err": err}


def traffic_from_profiles(kernel_stage, L, N):
    """DRAM bytes per launch of the dominant kernel, from the committed ncu
    summary (profiles/dram_traffic.txt: '<stage> <L> <N> <bytes>' lines)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        for ln in open(path):
            f = ln.split()
            if len(f) == 4 and f[0] == kernel_stage and int(f[1]) == L and int(f[2]) == N:
                return float(f[3])
    except Exception:
        pass
    return None


if __name__ == "__main__":
    a = args_()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
