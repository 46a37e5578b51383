"""Inverse -> forward round-trip error per band limit, FP64 path and split
precision (normwise relative error max|x - y| / max|y| against the input
coefficients).  Bounds: 1e-11 for the FP64 round trip, 1e-10 for each split
precision result against the FP64 path (its contract), 2e-10 for the split
round trip (two such stages composed).  L = 1024 also runs the
split-precision kernels past the shared-memory staging limit of the slicing
kernels (two-pass slicing) and reductions longer than 512 entries (seven-term
accumulator combination)."""
import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import params, rel_err

pytestmark = pytest.mark.gpu

CASES = [(8, 8), (64, 64), (256, 16), (512, 8), (1024, 4)]


@pytest.mark.parametrize("L,N", CASES, ids=[f"L{L}N{N}" for L, N in CASES])
def test_round_trip_per_band_limit(L, N, monkeypatch):
    import torch
    monkeypatch.setenv("SO3GPU_DIGIT_TABLE", "1")  # table-fed tensor-core kernels on the first call
    p = params(L, N)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 300 + i, "uniform")).cuda() for i in range(2)]
    f64 = ctx.inverse_batch(fls, p, "fp64")
    b64 = ctx.forward_batch(f64, p, "fp64")
    fmx = ctx.inverse_batch(fls, p, "mixed")
    bfw = ctx.forward_batch(f64, p, "mixed")  # split forward of the FP64 samples
    bmx = ctx.forward_batch(fmx, p, "mixed")  # split inverse then split forward
    torch.cuda.synchronize()
    fl, f64n, b64n, fmxn, bfwn, bmxn = ([x.cpu().numpy() for x in xs] for xs in (fls, f64, b64, fmx, bfw, bmx))
    e64 = max(rel_err(b, x) for b, x in zip(b64n, fl))
    e_inv = max(rel_err(a, b) for a, b in zip(fmxn, f64n))
    e_fwd = max(rel_err(a, b) for a, b in zip(bfwn, b64n))
    e_rt = max(rel_err(b, x) for b, x in zip(bmxn, fl))
    print(f"\nround trip L={L} N={N}: FP64 {e64:.2e}; split precision: inverse vs FP64 {e_inv:.2e}, "
          f"forward vs FP64 {e_fwd:.2e}, round trip {e_rt:.2e}")
    assert e64 < 1e-11
    assert e_inv < 1e-10 and e_fwd < 1e-10  # the split path's contract, per result
    assert e_rt < 2e-10  # two split stages composed
    assert so3.take_kernel_error() == 0
