#!/usr/bin/env python
"""Benchmark of the SO(3) Wigner transform path on B200.

Workload: complex signals at L=512, N=64, MW sampling, L0=0, padded storage,
negative-first n-order, all n, Risbo recursion, flmn real and imaginary
parts iid U(-1, 1) (seeded, per rank).  One transform unit = one inverse plus
one forward transform; the metric is units per second, split precision
against FP64.

  * headline step: inverse_batch + forward_batch of --batch signals (default
    16) with the int8 tensor-core (Ozaki split) contractions, FP64 everywhere
    else; its error against the FP64 path is measured on the same inputs;
  * "fp64": one FP64 inverse + forward per step (reference-exact path);
  * "e2e": end to end from pinned host buffers, copies included: signals
    streamed through the device API with the copies overlapped (value), and
    the synchronous drop-in so3_core_{inverse,forward}_via_ssht ("dropin").
Ranks run independent signals (weak scaling, no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]

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


_T0 = time.perf_counter()


def log(msg):
    """Progress of the legs on stderr (the JSON line goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--L", type=int, default=512)
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--batch", type=int, default=16,
                    help="signals per split-precision step (0: time the FP64 path only)")
    ap.add_argument("--serve", type=int, default=1500,
                    help="requests of the serving-trace sample (0: skip the serving leg)")
    ap.add_argument("--serve-rates", default="60,1000",
                    help="offered request rates of the serving leg (1/s, comma separated)")
    ap.add_argument("--serve-sweep", default="",
                    help="run only the serving sweep of the request trace: 20,000 requests at each of these offered "
                         "rates (comma separated), FP64 and split precision; prints one JSON line")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the split-precision leg's timed steps (the FP64 leg's with --batch 0) "
                         "with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--c3", type=int, default=512,
                    help="signals of the L=128, N=16 batched split-precision leg (0: skip it)")
    ap.add_argument("--c4", type=int, default=64,
                    help="kernels of the L=1024 directional-convolution leg (0: skip it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-full-unit", action="store_true",
                    help="also time one full CPU unit per process (no extrapolation; minutes at L=512, N=64)")
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
CPU_SAMPLE_N = 8  # the sampled unit's N: 2 * 8 - 1 = 15 of the n-planes


def _cpu_sample_worker(args):
    """One timed run of the reference's own CPU path (in a spawned process):
    so3_core_inverse_via_ssht + so3_core_forward_via_ssht, all n-planes, at
    band limit L and N (the bench's N for the full-unit check, CPU_SAMPLE_N
    for the bounded sample).  Returns wall seconds."""
    L, N, use_ref = args[:3]
    import ctypes

    import numpy as np
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from so3_b200 import synth
    p = O.params(L, N)
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
    return time.perf_counter() - t0


def cpu_unit_seconds(L, N, procs):
    """Per-process wall seconds of one full unit at (L, N), estimated from a
    complete transform at (L, CPU_SAMPLE_N) scaled by the number of n-planes
    (the per-plane work of the reference, one spin SHT and its share of the
    gamma FFT, hardly depends on n; checked against a full unit at L=512,
    N=64 with --cpu-full-unit)."""
    import multiprocessing as mp
    from oracle import oracle as O
    O.build()
    use_ref = O.ref() is not None
    ns = min(N, CPU_SAMPLE_N)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_sample_worker, [(L, ns, use_ref)] * procs)
    t = statistics.median(res)
    return t * (2 * N - 1) / (2 * ns - 1), t, use_ref


def cpu_full_unit_seconds(L, N, procs):
    """Per-process wall seconds of one FULL unit (all 2N-1 planes, no
    extrapolation), procs concurrent single-threaded processes: the check of
    the sampled estimate (minutes per process at L=512, N=64)."""
    import multiprocessing as mp
    from oracle import oracle as O
    O.build()
    use_ref = O.ref() is not None
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_sample_worker, [(L, N, use_ref)] * procs)
    return statistics.median(res)


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
    ns = min(a.N, CPU_SAMPLE_N)
    sample = (f"so3_core_inverse_via_ssht + so3_core_forward_via_ssht at L={a.L}, N={ns} (all {2 * ns - 1} "
              f"n-planes) per process, scaled by n-planes to N={a.N} ({2 * a.N - 1} planes); {procs} concurrent "
              f"single-threaded processes")
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
def fft_flops(n):
    """Nominal FFT flop count 5 n log2 n (the usual convention)."""
    return 5.0 * n * math.log2(n) if n > 1 else 0.0


def stage_work(L, N):
    """Algorithmic work per launch of every stage at (L, N), complex MW:
    (kind, amount, unit description)."""
    P, nb, ng, Pc = 2 * L - 1, L, 2 * N - 1, 1 << math.ceil(math.log2(4 * L - 3))
    planes = 2 * N - 1
    macs = contraction_macs(L, N)
    return {
        "inv_contract": ("fp64", 4.0 * macs, f"4 flops x {macs:.4g} complex-by-real MACs"),
        "fwd_contract": ("fp64", 4.0 * macs, f"4 flops x {macs:.4g} complex-by-real MACs"),
        "inv_beta": ("fp64", planes * L * fft_flops(P), f"{planes * L} DFTs of {P} (column pairs) at 5 n log2 n"),
        "inv_alpha": ("fp64", planes * nb * fft_flops(P), f"{planes * nb} DFTs of {P} at 5 n log2 n"),
        "fwd_alpha": ("fp64", planes * nb * fft_flops(P), f"{planes * nb} DFTs of {P} at 5 n log2 n"),
        "inv_gamma": ("fp64", nb * P * fft_flops(ng), f"{nb * P} DFTs of {ng} at 5 n log2 n"),
        "fwd_gamma": ("fp64", nb * P * fft_flops(ng), f"{nb * P} DFTs of {ng} at 5 n log2 n"),
        "fwd_beta_conv": ("fp64", planes * L * (fft_flops(P) + 2 * fft_flops(Pc)),
                          f"{planes * L} column pairs x (DFT {P} + 2 DFTs {Pc}) at 5 n log2 n"),
    }


def stage_bytes(L, N):
    """Compulsory HBM bytes of one launch of each FP64 stage (complex MW, one
    signal): every stage reads its input part once and writes its output part
    once.  Samples / row-major scratch: (2N-1) L (2L-1) complex; column-major
    spectra: (2N-1) (2L-1) L complex; coefficients: (2N-1) L^2 complex."""
    planes = 2 * N - 1
    part = planes * L * (2 * L - 1) * 16
    flmn = planes * L * L * 16
    return {"inv_contract": flmn + part, "inv_beta": 2 * part, "inv_alpha": 2 * part, "inv_gamma": 2 * part,
            "fwd_gamma": 2 * part, "fwd_alpha": 2 * part, "fwd_beta_conv": 2 * part, "fwd_contract": part + flmn,
            "mixed_inv_contract": flmn + part, "mixed_fwd_contract": part + flmn, "mixed_fwd_beta": 2 * part}


def hbm_peak():
    """HBM denominator: the measured-peaks file when present, else the
    recipe's fallback (6650 GB/s, an earlier STREAM-style copy on this pool)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        for k in ("hbm_gbs", "hbm_GBs", "hbm"):
            if k in d and float(d[k]) > 0:
                return float(d[k]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        pass
    return 6650.0, "fallback 6650 GB/s (no MEASURED_PEAKS.json)"


def elem_err(x, y, floor=1e-3):
    """Elementwise relative error max_i |x_i - y_i| / max(|y_i|, floor max|y|)
    of two device tensors (floor: a stated fraction of the largest magnitude,
    below which a relative error is ill-posed)."""
    ay = y.abs()
    den = ay.clamp(min=floor * float(ay.max().item()))
    return float(((x - y).abs() / den).max().item())


def mixed_tc_macs(L, N, fwd):
    """int8 multiply-adds the split-precision tensor-core kernel issues per
    group of 16 signals in one direction: per work item (pair (mu, nu), 64-row
    tile) nk reduction chunks of 64, each 2 x 28 digit products of
    128 x 64 x 32 (the inverse issues them as 2 x 10 MMAs with the table digits
    stacked along N; the multiply-adds are the same)."""
    import numpy as np
    T = 64
    MT = (L + T - 1) // T
    mu = np.arange(L)[:, None, None]
    nu = np.arange(N)[None, :, None]
    r0 = (np.arange(MT) * T)[None, None, :]
    lmin = np.maximum(mu, nu)
    if fwd:
        any_row = (r0 + T > lmin) & (r0 < L)
        kend = np.minimum(L, r0 + T)
        nk = np.where(any_row, (kend + T - 1) // T, 0)
    else:
        kstart = (np.maximum(lmin, r0) // T) * T
        nk = np.where(kstart < L, (L - kstart + T - 1) // T, 0)
    return int(nk.sum()) * 2 * 28 * 128 * 64 * 32


def split_stage_rooflines(per_launch_ms, L, N, B, int8_peak):
    """Tensor-pipe roofline of every split-precision stage of the headline
    step: int8 multiply-adds per launch (slicing kernel + tensor-core kernel)
    over the stage's measured launch time, against the measured int8 peak.
    per_launch_ms: {stage: ms per launch}; stages absent from it are left out."""
    groups = (B + 15) // 16
    macs = {"mixed_inv_contract": mixed_tc_macs(L, N, False) * groups,
            "mixed_fwd_contract": mixed_tc_macs(L, N, True) * groups,
            "mixed_fwd_beta": beta_tc_macs(L, N) * B}
    out = {}
    for k, m in macs.items():
        ms = per_launch_ms.get(k)
        if not ms or ms <= 0:
            continue
        tops = 2.0 * m / (ms * 1e-3) / 1e12
        out[k] = {"ms_per_launch": round(ms, 4), "int8_macs_per_launch": m, "achieved_tops": round(tops, 1),
                  "frac_int8_peak": round(tops / int8_peak, 4)}
    return out


def beta_tc_macs(L, N):
    """int8 multiply-adds of the split-precision forward beta stage per signal
    (complex MW): column tiles (2N-1 planes x 2 parity classes x ceil(L/64))
    x 64-row output tiles x L/64 reduction chunks, each 2 x 28 digit products
    of 128 x 64 x 32 (issued as 2 x 10 MMAs, N up to 256)."""
    T = 64
    nc = (L + T - 1) // T
    tiles = (2 * N - 1) * 2 * nc
    return tiles * nc * nc * 2 * 28 * 128 * 64 * 32


def timed_steps(step, steps, warmup, stream, ctx, so3, sdist, local, world, profile=False):
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        sdist.barrier()
    ctx.stage_timing(True)
    ctx.stage_times()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    launches0 = so3.launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if profile:
            torch.cuda.profiler.start()
        evs[0].record(stream)
        for i in range(steps):
            step()
            evs[i + 1].record(stream)
        torch.cuda.synchronize()
        if profile:
            torch.cuda.profiler.stop()
    launches = so3.launch_count() - launches0
    stages = ctx.stage_times()
    ctx.stage_timing(False)
    total_ms = evs[0].elapsed_time(evs[-1])
    lat = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
    total_ms = sdist.max_over_ranks(total_ms, device=f"cuda:{local}")
    return {"total_ms": total_ms, "lat": lat, "launches": launches, "stages": stages, "clocks": clk.summary()}


def pct(lat, q):
    s = sorted(lat)
    return s[min(len(s) - 1, max(0, math.ceil(q * len(s)) - 1))]


def serving_child(n, rate, seed, prec, device, max_batch, shapes, warm=False, timeout=420):
    """One serving measurement in a child process (its own CUDA context and
    tables), killed after `timeout` seconds: a stalled trace cannot hold up
    the rest of the bench.  warm: one untimed pass of the same trace first."""
    code = ("import json,sys; sys.path.insert(0, %r); from so3_b200 import serve as s; "
            "kw=dict(seed=%d, precision=%r, device=%d, max_batch=%d, shapes=%r); "
            "%s print(json.dumps(s.serving_run(%d, %r, **kw)))"
            % (ROOT, seed, prec, device, max_batch, shapes,
               ("s.serving_run(%d, %r, **kw); " % (n, rate)) if warm else "", n, rate))
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"timed_out_s": timeout, "requests": n, "offered_rate_rps": rate, "precision": prec}
    if r.returncode != 0:
        return {"failed": r.stderr.strip().splitlines()[-1:] if r.stderr else ["no output"], "requests": n,
                "offered_rate_rps": rate, "precision": prec}
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_serve_sweep(a):
    """Config C5 at its stated size: 20,000 seeded requests (60 % inverse /
    40 % forward complex MW, L log-uniform in [16, 1024], N uniform in
    [1, min(L, 64)], U(-1,1) inputs, Poisson arrivals) at each offered rate,
    FP64 and split precision, 120 GB admission budget: throughput, p50 / p99
    latency, mean unit size."""
    rates = [float(x) for x in a.serve_sweep.split(",") if x]
    rows = []
    for rate in rates:
        row = {"offered_rate_rps": rate}
        for prec in ("fp64", "mixed"):
            row[prec] = serving_child(20000, rate, 11, prec, 0, 16, None, timeout=1500)
        rows.append(row)
        print(json.dumps({"partial": row}), file=sys.stderr, flush=True)
    print(json.dumps({"serving_sweep": rows, "requests_per_rate": 20000,
                      "trace": "60% inverse / 40% forward, complex MW, L log-uniform [16, 1024], "
                               "N uniform [1, min(L, 64)], U(-1,1), Poisson, 120 GB budget, 8 slots, units <= 16"}),
          flush=True)


def run_ours(a):
    import torch
    if a.serve_sweep:
        run_serve_sweep(a)
        return

    import so3_b200 as so3
    from so3_b200 import dist as sdist
    from so3_b200 import synth

    info = sdist.rank_info()
    world, rank, local = info.world, info.rank, info.local
    torch.cuda.set_device(local)
    sdist.init("nccl" if world > 1 else None, timeout_s=120)
    dev = f"cuda:{local}"

    L, N, B = a.L, a.N, a.batch
    p = so3.SO3Parameters(L=L, N=N, L0=0, sampling_scheme=0, n_order=1, storage=0, n_mode=0, dl_method=0)
    stream = torch.cuda.current_stream()
    ctx = so3.Context(local, stream=stream)
    ctx.prepare(p)
    from so3_b200 import peaks
    log("probes")
    fp64_peak = peaks.fp64_tflops(local)
    int8_peak = peaks.int8_mma_tops(local)
    probes = {"fp64_fma_tflops": fp64_peak, "fp64_dmma_tflops": peaks.dmma_tflops(local),
              "int8_tcgen05_tops": int8_peak, "hbm_copy_gbs": peaks.hbm_copy_gbs(local)}

    log("fp64 leg")
    # ---- plain FP64 path, one signal per step
    fl_host = synth.gen_flmn(p, sdist.signal_seed(1000, rank, 0), "uniform")
    d_flmn = torch.from_numpy(fl_host).to(dev)
    d_f = torch.empty(so3.f_size(p), dtype=torch.complex128, device=dev)
    d_back = torch.empty(so3.flmn_size(p), dtype=torch.complex128, device=dev)

    def step64():
        ctx.inverse(d_flmn, p, out=d_f)
        ctx.forward(d_f, p, out=d_back)

    r64 = timed_steps(step64, a.steps, a.warmup, stream, ctx, so3, sdist, local, world, a.profile_region and B == 0)
    fp64_value = sdist.job_throughput(world * a.steps, r64["total_ms"] / 1e3)
    rt_err = float(((d_back - d_flmn).abs().max() / d_flmn.abs().max()).item())
    log("fp64 leg, other contraction engine")
    # the other FP64 contraction engine (FP64 tensor cores <-> FMA kernels), same step, same inputs
    other = "0" if os.environ.get("SO3GPU_FP64_MMA", "1") != "0" else "1"
    prev = os.environ.get("SO3GPU_FP64_MMA")
    os.environ["SO3GPU_FP64_MMA"] = other
    d_back2 = torch.empty_like(d_back)
    ref_back = d_back.clone()

    def step64b():
        ctx.inverse(d_flmn, p, out=d_f)
        ctx.forward(d_f, p, out=d_back2)

    r64b = timed_steps(step64b, a.steps, a.warmup, stream, ctx, so3, sdist, local, world)
    torch.cuda.synchronize()
    fp64_alt = {"engine": "fp64 tensor cores (mma.sync m8n8k4)" if other == "1" else "fp64 FMA kernels",
                "value": sdist.job_throughput(world * a.steps, r64b["total_ms"] / 1e3),
                "ms_per_step": r64b["total_ms"] / a.steps,
                "stage_ms": {k: round(v[0] / v[1], 4) for k, v in r64b["stages"].items()},
                "rel_diff_vs_default_engine": float(((d_back2 - ref_back).abs().max() / ref_back.abs().max()).item())}
    if prev is None:
        del os.environ["SO3GPU_FP64_MMA"]
    else:
        os.environ["SO3GPU_FP64_MMA"] = prev
    del d_back2, ref_back
    del d_back

    log("split-precision leg")
    # ---- split-precision batch path: B signals per step
    mixed = None
    headline = {"value": fp64_value, "run": r64, "units_per_step": 1, "precision": "fp64"}
    if B > 0:
        fls = [d_flmn] + [torch.from_numpy(synth.gen_flmn(p, sdist.signal_seed(1000, rank, i), "uniform")).to(dev)
                          for i in range(1, B)]
        fs = [torch.empty(so3.f_size(p), dtype=torch.complex128, device=dev) for _ in range(B)]
        backs = [torch.zeros(so3.flmn_size(p), dtype=torch.complex128, device=dev) for _ in range(B)]

        def stepmx():
            ctx.inverse_batch(fls, p, "mixed", outs=fs)
            ctx.forward_batch(fs, p, "mixed", outs=backs)

        rmx = timed_steps(stepmx, a.steps, a.warmup, stream, ctx, so3, sdist, local, world, a.profile_region)
        mixed_value = sdist.job_throughput(world * a.steps * B, rmx["total_ms"] / 1e3)
        # error of the split path against the FP64 path on the same inputs
        err_f = err_fl = err_rt = ee_f = ee_fl = 0.0
        for i in range(B):
            ctx.inverse(fls[i], p, out=d_f)
            torch.cuda.synchronize()
            err_f = max(err_f, float(((fs[i] - d_f).abs().max() / d_f.abs().max()).item()))
            ee_f = max(ee_f, elem_err(fs[i], d_f))
            ref = ctx.forward(fs[i], p)
            torch.cuda.synchronize()
            err_fl = max(err_fl, float(((backs[i] - ref).abs().max() / ref.abs().max()).item()))
            ee_fl = max(ee_fl, elem_err(backs[i], ref))
            err_rt = max(err_rt, float(((backs[i] - fls[i]).abs().max() / fls[i].abs().max()).item()))
            del ref
        del fls, fs, backs  # release the batch before the end-to-end and serving legs
        torch.cuda.empty_cache()
        mixed = {"value": mixed_value, "unit": UNIT, "batch": B, "ms_per_step": rmx["total_ms"] / a.steps,
                 "over_fp64": mixed_value / fp64_value,
                 "rel_err_vs_fp64": {"samples": err_f, "coefficients": err_fl, "max": max(err_f, err_fl),
                                     "definition": "normwise max|x-y| / max|y| over each signal, max over signals"},
                 "elementwise_rel_err_vs_fp64": {
                     "samples": ee_f, "coefficients": ee_fl, "max": max(ee_f, ee_fl),
                     "definition": "max_i |x_i-y_i| / max(|y_i|, 1e-3 max|y|): elementwise, floor 1e-3 of the "
                                   "largest magnitude"},
                 "roundtrip_rel_err": err_rt}
        headline = {"value": mixed_value, "run": rmx, "units_per_step": B, "precision": "mixed"}

    run = headline["run"]
    ups = headline["units_per_step"]
    stages = run["stages"]
    per_signal = {k: v[0] / (a.steps * ups) for k, v in stages.items()}  # ms per transform unit
    per_launch = {k: v[0] / v[1] for k, v in stages.items()}

    # ---- roofline of the dominant kernel of the headline step
    work = stage_work(L, N)
    dom = max(per_signal, key=per_signal.get)
    t_launch = per_launch[dom] / 1e3
    if dom.startswith("mixed"):
        if dom == "mixed_fwd_beta":
            macs = beta_tc_macs(L, N) * B
        else:
            macs = mixed_tc_macs(L, N, dom == "mixed_fwd_contract") * ((B + 15) // 16)
        ops = 2.0 * macs
        achieved = ops / t_launch / 1e12
        roof = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOP/s",
                "frac": achieved / int8_peak,
                "peak_source": "tcgen05.mma kind::i8 128x256x32 back-to-back on this GPU "
                               "(so3_b200/peaks: tcgen05 probe); nominal int8 dense peak 4500 TOP/s",
                "algorithmic": f"{macs:.4g} int8 MACs per launch (28 digit products, batch {B}, "
                               f"stage = slicing kernel + tensor-core kernel; int8 peak measured with tcgen05)"}
    else:
        kind, amount, desc = work[dom]
        achieved = amount / t_launch / 1e12
        roof = {"kernel": dom, "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak,
                "peak_source": "FP64 FMA-chain microbenchmark on this GPU (so3_b200/peaks); the "
                               "measured-peaks file has no FP64 figure", "algorithmic": desc + " per launch"}
    roof["traffic"] = traffic_from_profiles(dom, L, N)
    roof["traffic_source"] = "profiles/dram_traffic.txt (ncu dram__bytes_read.sum + dram__bytes_write.sum)"
    roof["avg_ms"] = per_launch[dom]
    if dom.startswith("mixed"):
        # FP64-equivalent: the flops of the FP64 algorithm the int8 products replace
        if dom == "mixed_fwd_beta":
            planes = 2 * N - 1
            fl64 = 2.0 * planes * (2 * L - 1) * 2 * L * L * B  # dense real map R_s on re/im of every column
            what = "dense beta map R_s: 2 flops x (2N-1)(2L-1) columns x re/im x L x L, per signal"
        else:
            fl64 = 4.0 * contraction_macs(L, N) * B
            what = "4 flops x complex-by-real MACs of the contraction, per signal"
        roof["fp64_equivalent"] = {"achieved": fl64 / t_launch / 1e12, "unit": "TFLOP/s",
                                   "fp64_peak": fp64_peak, "frac_of_fp64_peak": fl64 / t_launch / 1e12 / fp64_peak,
                                   "algorithmic": what}

    if dom.startswith("mixed"):
        try:
            roof["split_stages"] = split_stage_rooflines(per_launch, L, N, B, int8_peak)
        except Exception as e:  # a reporting helper never costs the bench line
            roof["split_stages"] = {"error": str(e)}

    # per-stage HBM roofline of every stage of the headline step and of the FP64 step
    hbm, hbm_src = hbm_peak()
    sb = stage_bytes(L, N)

    def stage_roof(stg, units):
        out = {}
        for k, (tot, cnt) in stg.items():
            if k not in sb or cnt == 0:
                continue
            ms = tot / cnt
            by = sb[k] * units(k)
            out[k] = {"ms_per_launch": round(ms, 4), "bytes_per_launch": by,
                      "gbs": round(by / (ms * 1e-3) / 1e9, 1), "frac_hbm": round(by / (ms * 1e-3) / 1e9 / hbm, 3)}
        return out

    hbm_stages = {"peak_gbs": hbm, "peak_source": hbm_src, "fp64_step": stage_roof(r64["stages"], lambda k: 1)}
    if mixed:
        hbm_stages["split_step"] = stage_roof(run["stages"], lambda k: B if k.startswith("mixed") else 1)

    log("C3 leg")
    # ---- config C3: 512 signals, L=128, N=16, Gaussian (l+1)^-2, split vs FP64
    c3 = None
    if a.c3 > 0 and B > 0:
        c3 = run_c3(so3, synth, a.c3, rank, dev, a.steps, a.warmup, stream, sdist, local, world)

    log("C4 leg")
    # ---- config C4: one S^2 signal at L=1024 convolved with kernels (N=8), inverse to samples
    c4 = None
    if a.c4 > 0 and B > 0:
        c4 = run_c4(so3, synth, a.c4, rank, dev, stream, sdist, local, world)

    log("e2e leg")
    # ---- end to end through the drop-in C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(so3, p, fl_host, a.steps, local, world)
        e2e["dropin"] = run_e2e_dropin(so3, p, fl_host, min(a.steps, 3), local, world)

    # ---- serving: a sample of the request trace (inverse 60 % / forward 40 %, complex MW, L log-uniform
    # in [16, 1024], N uniform in [1, min(L, 64)], U(-1,1) inputs, Poisson arrivals), FP64 and split
    serving = None
    if a.serve > 0:
        from so3_b200 import serve as sserve
        ctx.close()  # the batch workspace
        del d_flmn, d_f
        torch.cuda.empty_cache()
        rates = [float(x) for x in a.serve_rates.split(",") if x]
        serving = {"trace": f"{a.serve} requests per rate, seed {rank + 11}, Poisson arrivals at each offered rate, "
                            f"L log-uniform [16, 1024], N uniform [1, min(L, 64)], 60% inverse / 40% forward, "
                            f"complex MW, 120 GB budget (resident tables and buffers included), 8 slots, "
                            f"units of up to 16 (split precision across geometries)", "by_rate": []}
        for rate in rates:
            row = {"offered_rate_rps": rate}
            for prec in ("fp64", "mixed"):
                log(f"serving {prec} at {rate:g}/s")
                row[prec] = serving_child(a.serve, rate, rank + 11, prec, local, 16, None)
            serving["by_rate"].append(row)
        # recurring geometries offered as a burst: split-precision requests batch (up to 8 per launch)
        shapes = [(512, 16), (256, 32), (128, 64)]
        serving["recurring"] = {"trace": f"256 requests, (L, N) uniform over {shapes}, 60% inverse / 40% forward, "
                                         f"Poisson 1000/s offered, batches of up to 8; measured after one untimed "
                                         f"pass of the same trace (resident tables built)"}
        for prec in ("fp64", "mixed"):
            log(f"serving recurring {prec}")
            serving["recurring"][prec] = serving_child(256, 1000.0, rank + 21, prec, local, 8, shapes, warm=True)

    cpu = None
    log("cpu baseline")
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            procs = cpu_procs(L, N)
            unit_s, samp_s, use_ref = cpu_unit_seconds(L, N, procs)
            cpu = {"value": procs / unit_s, "unit": UNIT, "cores": procs,
                   "kind": "reference" if use_ref else "port",
                   "sample": f"inverse+forward at L={L}, N={min(N, CPU_SAMPLE_N)} (all {2 * min(N, CPU_SAMPLE_N) - 1} "
                             f"n-planes, {samp_s:.1f} s per process), scaled by n-planes to N={N}; {procs} "
                             f"concurrent single-threaded processes",
                   "seconds_per_unit_per_process": unit_s}
            if a.cpu_full_unit:
                log("cpu full unit")
                full_s = cpu_full_unit_seconds(L, N, procs)
                cpu["full_unit_check"] = {"seconds_per_unit_per_process": full_s, "value": procs / full_s,
                                          "estimate_over_full": unit_s / full_s,
                                          "what": "one full inverse+forward (all planes) per process, no "
                                                  "extrapolation, same processes"}
        except Exception as ex:  # the CPU baseline never blocks the GPU line
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        lat = run["lat"]
        line = {"metric": METRIC, "value": headline["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": run["total_ms"] / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "int8 Ozaki split (7 x 7-bit digits, 49-bit fixed point, exact int32 sums) + f64"
                if mixed else "f64", "data": "synthetic",
                "config": dict(workload(L, N), batch=B if mixed else 1,
                               step=f"inverse_batch + forward_batch of {B} signals, split-precision contractions"
                               if mixed else "one inverse + one forward, FP64"),
                "precision": headline["precision"],
                "mixed": mixed,
                "fp64_other_engine": fp64_alt,
                "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": r64["total_ms"] / a.steps,
                         "roundtrip_rel_err": rt_err,
                         "stage_ms": {k: round(v[0] / v[1], 4) for k, v in r64["stages"].items()},
                         "latency_ms": {"p50": statistics.median(r64["lat"]), "p99": pct(r64["lat"], 0.99)}},
                "latency_ms": {"p50": statistics.median(lat), "p99": pct(lat, 0.99)},
                "stage_ms_per_transform": {k: round(v, 4) for k, v in per_signal.items()},
                "gpu_launches": int(run["launches"]), "roofline": roof, "stage_hbm": hbm_stages,
                "probes": probes,
                "c3": c3, "c4": c4, "e2e": e2e, "cpu_baseline": cpu,
                "serving": serving,
                "clocks": run["clocks"]}
        print(json.dumps(line), flush=True)
    sdist.finalize()


def run_c3(so3, synth, nsig, rank, dev, steps, warmup, stream, sdist, local, world):
    """Batched split precision at its stated size: nsig complex signals at
    L=128, N=16, MW, padded, Risbo, complex Gaussian coefficients with variance
    (l+1)^-2; one step = inverse + forward of every signal, split precision
    (one batch call per direction) against FP64 (signal by signal), with the
    split path's error against FP64 on every signal."""
    import torch
    L, N = 128, 16
    p = so3.SO3Parameters(L=L, N=N, L0=0, sampling_scheme=0, n_order=1, storage=0, n_mode=0, dl_method=0)
    ctx = so3.Context(local, stream=stream)
    fls = [torch.from_numpy(synth.gen_flmn(p, sdist.signal_seed(5000, rank, i), "gauss")).to(dev)
           for i in range(nsig)]
    fs = [torch.empty(so3.f_size(p), dtype=torch.complex128, device=dev) for _ in range(nsig)]
    backs = [torch.zeros(so3.flmn_size(p), dtype=torch.complex128, device=dev) for _ in range(nsig)]
    f64 = [torch.empty_like(fs[0]) for _ in range(nsig)]
    b64 = [torch.zeros_like(backs[0]) for _ in range(nsig)]

    def step_mx():
        ctx.inverse_batch(fls, p, "mixed", outs=fs)
        ctx.forward_batch(fs, p, "mixed", outs=backs)

    def step_64():
        ctx.inverse_batch(fls, p, "fp64", outs=f64)
        ctx.forward_batch(f64, p, "fp64", outs=b64)

    r64 = timed_steps(step_64, steps, warmup, stream, ctx, so3, sdist, local, world)
    rmx = timed_steps(step_mx, steps, warmup, stream, ctx, so3, sdist, local, world)
    v64 = sdist.job_throughput(world * steps * nsig, r64["total_ms"] / 1e3)
    vmx = sdist.job_throughput(world * steps * nsig, rmx["total_ms"] / 1e3)
    # split forward on the FP64 samples, so each direction's error is its own
    ctx.forward_batch(f64, p, "mixed", outs=backs)
    torch.cuda.synchronize()
    en_f = en_b = ee_f = ee_b = 0.0
    for i in range(nsig):
        en_f = max(en_f, float(((fs[i] - f64[i]).abs().max() / f64[i].abs().max()).item()))
        ee_f = max(ee_f, elem_err(fs[i], f64[i]))
        en_b = max(en_b, float(((backs[i] - b64[i]).abs().max() / b64[i].abs().max()).item()))
        ee_b = max(ee_b, elem_err(backs[i], b64[i]))
    out = {"workload": f"{nsig} complex signals, L={L}, N={N}, MW, padded, Risbo, Gaussian (l+1)^-2",
           "mixed": vmx, "fp64": v64, "unit": UNIT, "over_fp64": vmx / v64,
           "ms_per_step": {"mixed": rmx["total_ms"] / steps, "fp64": r64["total_ms"] / steps},
           "rel_err_vs_fp64": {"samples": en_f, "coefficients": en_b},
           "elementwise_rel_err_vs_fp64": {"samples": ee_f, "coefficients": ee_b, "floor": 1e-3}}
    del fls, fs, backs, f64, b64
    ctx.close()
    torch.cuda.empty_cache()
    return out


def run_c4(so3, synth, nker, rank, dev, stream, sdist, local, world, chunk=16, steps=2, warmup=2):
    """Directional convolution at L=1024: one S^2 signal flm (complex
    Gaussian, variance (l+1)^-2) convolved with nker kernels glm (complex
    Gaussian for |m| < 8, zero otherwise) by so3_conv_s2toso3_harmonic_
    convolution (N=8), each result inverse-transformed to MW samples; the
    kernels run in chunks of `chunk` (so3gpu_s2toso3_inverse_batch), FP64
    against split precision (h built inside the contraction's operand load).
    One step = all nker kernels; value in kernels/s."""
    import torch
    L, N = 1024, 8
    hp = so3.SO3Parameters(L=L, N=N, L0=0, sampling_scheme=0, n_order=1, storage=0, n_mode=0, dl_method=0)
    ctx = so3.Context(local, stream=stream)
    flm = torch.from_numpy(synth.gen_flm(L, sdist.signal_seed(7000, rank, 0), "gauss")).to(dev)
    glms = [torch.from_numpy(synth.gen_flm(L, sdist.signal_seed(7001, rank, k), "gauss", mmax=N - 1)).to(dev)
            for k in range(nker)]
    outs = [torch.empty(so3.f_size(hp), dtype=torch.complex128, device=dev) for _ in range(chunk)]
    ref = [torch.empty(so3.f_size(hp), dtype=torch.complex128, device=dev) for _ in range(chunk)]

    def step(prec):
        for c0 in range(0, nker, chunk):
            g = glms[c0:c0 + chunk]
            ctx.s2toso3_inverse_batch(hp, flm, g, prec, outs=outs[:len(g)])

    res = {}
    for prec in ("fp64", "mixed"):
        r = timed_steps(lambda: step(prec), steps, warmup, stream, ctx, so3, sdist, local, world)
        res[prec] = sdist.job_throughput(world * steps * nker, r["total_ms"] / 1e3)
    # error of split against FP64 on the first chunk
    g = glms[:chunk]
    ctx.s2toso3_inverse_batch(hp, flm, g, "fp64", outs=ref[:len(g)])
    ctx.s2toso3_inverse_batch(hp, flm, g, "mixed", outs=outs[:len(g)])
    torch.cuda.synchronize()
    en = max(float(((o - r_).abs().max() / r_.abs().max()).item()) for o, r_ in zip(outs[:len(g)], ref))
    ee = max(elem_err(o, r_) for o, r_ in zip(outs[:len(g)], ref))
    out = {"workload": f"flm L={L} (Gaussian (l+1)^-2) convolved with {nker} kernels (|m| < {N}), N={N}, "
                       f"inverse to MW samples, chunks of {chunk}",
           "unit": "kernels/s", "fp64": res["fp64"], "mixed": res["mixed"], "over_fp64": res["mixed"] / res["fp64"],
           "steps": steps, "warmup": warmup,
           "rel_err_vs_fp64": en, "elementwise_rel_err_vs_fp64": ee}
    del outs, ref, glms, flm
    ctx.close()
    torch.cuda.empty_cache()
    return out


def run_e2e_dropin(so3, p, fl_host, steps, local, world):
    """Same metric through so3_core_{inverse,forward}_via_ssht on pinned host
    buffers, one synchronous call after the other: every step copies flmn and f
    host->device and f and flmn back."""
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
            "d2h_bytes_per_step": nb_f + nb_fl, "steps": steps,
            "api": "so3_core_inverse_via_ssht + so3_core_forward_via_ssht (host pointers, pinned, synchronous)",
            "roundtrip_rel_err": err}


def run_e2e(so3, p, fl_host, steps, local, world, depth=3):
    """The metric end to end from pinned host memory through the library's
    device API (so3_b200.Context, FP64 path), signals streamed: one step = one
    unit = copy flmn host->device, inverse, copy f device->host, copy that host
    f back host->device, forward, copy flmn device->host; all copies of every
    step are inside the timed region.  Copies run on their own streams (one per
    direction) and overlap the transforms and the other direction's copies of
    neighbouring units (`depth` device buffer sets in rotation); issue order
    A(0) A(1) B(0) A(2) B(1) ..., A = upload + inverse + download of f, B =
    re-upload of f + forward + download of flmn.  Wall clock over the whole
    stream, synchronised on both sides, max over ranks."""
    import numpy as np
    import torch

    from so3_b200 import dist as sdist
    dev = f"cuda:{local}"
    nfl, nf = so3.flmn_size(p), so3.f_size(p)
    units = max(steps, 16)
    comp, up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ctx = so3.Context(local, stream=comp)
    ctx.prepare(p)
    fl_pin = torch.from_numpy(fl_host).pin_memory()
    f_pin = [torch.empty(nf, dtype=torch.complex128).pin_memory() for _ in range(depth)]
    back_pin = [torch.empty(nfl, dtype=torch.complex128).pin_memory() for _ in range(depth)]
    d_fl = [torch.empty(nfl, dtype=torch.complex128, device=dev) for _ in range(depth)]
    d_f = [torch.empty(nf, dtype=torch.complex128, device=dev) for _ in range(depth)]
    d_fin = [torch.empty(nf, dtype=torch.complex128, device=dev) for _ in range(depth)]
    d_back = [torch.empty(nfl, dtype=torch.complex128, device=dev) for _ in range(depth)]
    free = [None] * depth  # event: slot's last download done

    def stage_a(s):
        i = s % depth
        with torch.cuda.stream(up):
            if free[i] is not None:
                up.wait_event(free[i])
            d_fl[i].copy_(fl_pin, non_blocking=True)
            e = torch.cuda.Event()
            e.record(up)
        comp.wait_event(e)
        ctx.inverse(d_fl[i], p, out=d_f[i])
        e = torch.cuda.Event()
        e.record(comp)
        with torch.cuda.stream(down):
            down.wait_event(e)
            f_pin[i].copy_(d_f[i], non_blocking=True)
            e = torch.cuda.Event()
            e.record(down)
        return e

    def stage_b(s, got_f):
        i = s % depth
        with torch.cuda.stream(up):
            up.wait_event(got_f)
            d_fin[i].copy_(f_pin[i], non_blocking=True)
            e = torch.cuda.Event()
            e.record(up)
        comp.wait_event(e)
        ctx.forward(d_fin[i], p, out=d_back[i])
        e = torch.cuda.Event()
        e.record(comp)
        with torch.cuda.stream(down):
            down.wait_event(e)
            back_pin[i].copy_(d_back[i], non_blocking=True)
            free[i] = torch.cuda.Event()
            free[i].record(down)

    def run(n):
        pend = stage_a(0)
        for s in range(1, n):
            nxt = stage_a(s)
            stage_b(s - 1, pend)
            pend = nxt
        stage_b(n - 1, pend)

    run(depth)  # warm-up: buffers, plans, pinned-memory registration
    torch.cuda.synchronize()
    if world > 1:
        sdist.barrier()
    t0 = time.perf_counter()
    run(units)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    el = sdist.max_over_ranks(el, device=dev)
    last = (units - 1) % depth
    err = float(np.abs(back_pin[last].numpy() - fl_host).max() / np.abs(fl_host).max())
    ctx.close()
    out = {"value": world * units / el, "unit": UNIT, "h2d_bytes_per_step": 16 * (nfl + nf),
           "d2h_bytes_per_step": 16 * (nf + nfl), "steps": units, "precision": "fp64",
           "api": "so3_b200.Context.inverse / forward (so3gpu_inverse / so3gpu_forward) on device buffers, "
                  "pinned host buffers copied on two copy streams, units streamed",
           "roundtrip_rel_err": err}
    del d_fl, d_f, d_fin, d_back
    torch.cuda.empty_cache()
    return out


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
