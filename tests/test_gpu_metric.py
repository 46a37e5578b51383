"""Parity at the metric geometry (complex MW, L=512, N=64, padded,
negative-first, Risbo, U(-1,1) coefficients).

* FP64 GPU path against the oracle on the planes n = +-63 (n_mode=MAXIMUM:
  the full L=512 contraction and DFT lengths 1023 / 127 at the planes with
  the largest |n|), inverse and forward (forward on the oracle's samples):
  1e-12 normwise relative error, as every FP64 parity test.
* Split-precision batch (3 signals, all 127 planes) against the FP64 path on
  the same inputs: <= 1e-10 normwise relative error, the split path's stated
  contract.  The elementwise relative error with a floor at 1e-3 of the
  largest magnitude (tests.helpers.rel_err_elem) is checked beside it."""
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import oparams, params, rel_err, rel_err_elem

pytestmark = pytest.mark.gpu


def test_fp64_metric_geometry_max_planes_against_oracle(O):
    p = params(512, 64, mode=3)
    op = oparams(O, p)
    fl = synth.gen_flmn(p, 4242, "uniform")
    f_gpu = so3.inverse(fl, p)
    f_ref = O.inverse(fl, op)
    assert rel_err(f_gpu, f_ref) < 1e-12
    assert rel_err_elem(f_gpu, f_ref) < 1e-9
    fl_gpu = so3.forward(f_ref, p)
    fl_ref = O.forward(f_ref, op)
    assert rel_err(fl_gpu, fl_ref) < 1e-12
    assert rel_err_elem(fl_gpu, fl_ref) < 1e-9
    assert rel_err(fl_gpu, fl) < 1e-11  # round trip


def test_split_metric_geometry_against_fp64(monkeypatch):
    import torch
    monkeypatch.setenv("SO3GPU_DIGIT_TABLE", "1")  # the table-fed kernels of the bench step
    p = params(512, 64)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 900 + i, "uniform")).cuda() for i in range(3)]
    f64 = ctx.inverse_batch(fls, p, "fp64")
    fmx = ctx.inverse_batch(fls, p, "mixed")
    b64 = ctx.forward_batch(f64, p, "fp64")
    bmx = ctx.forward_batch(f64, p, "mixed")
    torch.cuda.synchronize()
    assert so3.take_kernel_error() == 0
    for i in range(3):
        x, y = fmx[i].cpu().numpy(), f64[i].cpu().numpy()
        assert rel_err(x, y) <= 1e-10
        assert rel_err_elem(x, y) <= 1e-7
        x, y = bmx[i].cpu().numpy(), b64[i].cpu().numpy()
        assert rel_err(x, y) <= 1e-10
        assert rel_err_elem(x, y) <= 1e-7
    del fmx, bmx, b64, f64
    ctx.close()
    torch.cuda.empty_cache()
