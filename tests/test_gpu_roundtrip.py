"""Inverse -> forward round-trip error per band limit, FP64 path and split
precision (normwise relative error max|x - y| / max|y| against the input
coefficients).  Bounds: 1e-11 for FP64 (measured 1e-14 .. 4e-13), 1e-10 for
split precision (its contract against FP64).  L = 1024 also runs the
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
    bmx = ctx.forward_batch(fmx, p, "mixed")
    torch.cuda.synchronize()
    e64 = max(rel_err(b.cpu().numpy(), x.cpu().numpy()) for b, x in zip(b64, fls))
    emx = max(rel_err(b.cpu().numpy(), x.cpu().numpy()) for b, x in zip(bmx, fls))
    print(f"\nround trip L={L} N={N}: FP64 {e64:.2e}, split precision {emx:.2e}")
    assert e64 < 1e-11
    assert emx < 1e-10
    assert so3.take_kernel_error() == 0
