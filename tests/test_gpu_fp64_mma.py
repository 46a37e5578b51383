"""FP64 contraction on the FP64 tensor cores (mma.sync m8n8k4 f64, the
default for complex signals; SO3GPU_FP64_MMA=0 selects the FMA kernels)
against the oracle and against the FP64 FMA kernels, on
the same seeded inputs: 1e-12 normwise relative error, as every FP64 parity
test."""
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import oparams, params, rel_err

pytestmark = pytest.mark.gpu

CASES = [dict(L=64, N=64), dict(L=17, N=3, L0=5), dict(L=24, N=9, storage=1, order=0), dict(L=20, N=6, mode=1),
         dict(L=20, N=6, mode=3), dict(L=33, N=5, sampling=1, method=1), dict(L=1, N=1), dict(L=2, N=2),
         dict(L=70, N=4, mode=4)]


@pytest.mark.parametrize("kw", CASES, ids=[str(i) for i in range(len(CASES))])
def test_fp64_mma_inverse_against_oracle_and_fma(O, monkeypatch, kw):
    kw = dict(kw)
    p = params(kw.pop("L"), kw.pop("N"), **kw)
    fl = synth.gen_flmn(p, 313)
    monkeypatch.setenv("SO3GPU_FP64_MMA", "0")
    f_fma = so3.inverse(fl, p)
    monkeypatch.setenv("SO3GPU_FP64_MMA", "1")
    f_mma = so3.inverse(fl, p)
    assert rel_err(f_mma, f_fma) < 1e-13
    assert rel_err(f_mma, O.inverse(fl, oparams(O, p))) < 1e-12
    f_ref = O.inverse(fl, oparams(O, p))
    monkeypatch.setenv("SO3GPU_FP64_MMA", "0")
    b_fma = so3.forward(f_ref, p)
    monkeypatch.setenv("SO3GPU_FP64_MMA", "1")
    b_mma = so3.forward(f_ref, p)
    assert rel_err(b_mma, b_fma) < 1e-13
    assert rel_err(b_mma, O.forward(f_ref, oparams(O, p))) < 1e-12
    assert rel_err(so3.forward(f_mma, p), fl) < 1e-11


def test_fp64_mma_metric_geometry_max_planes(O, monkeypatch):
    monkeypatch.setenv("SO3GPU_FP64_MMA", "1")
    p = params(512, 64, mode=3)
    fl = synth.gen_flmn(p, 4243)
    f_ref = O.inverse(fl, oparams(O, p))
    assert rel_err(so3.inverse(fl, p), f_ref) < 1e-12
    assert rel_err(so3.forward(f_ref, p), O.forward(f_ref, oparams(O, p))) < 1e-12
