"""DFT-stage autotuner: every kernel variant of a stage computes the same
per-sequence arithmetic, so pinning any variant must reproduce the default
results bit for bit; tuning must pick variants that exist."""
import ctypes

import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import params

pytestmark = pytest.mark.gpu


def _vars(lib, p, values):
    arr = (ctypes.c_int * 8)(*values)
    assert lib.so3gpu_set_stage_variants(0, ctypes.byref(p.to_struct()), arr) == 0


@pytest.mark.parametrize("L,N", [(512, 2), (64, 64)])
def test_every_variant_gives_identical_results(L, N):
    import torch
    lib = so3._lib.load()
    p = params(L, N)
    fl = torch.from_numpy(synth.gen_flmn(p, 21)).cuda()
    ctx = so3.Context(0)
    outs = []
    for v in (0, 1, 2, 3):
        _vars(lib, p, [v] * 8)
        f = ctx.inverse(fl, p)
        back = ctx.forward(f, p)
        torch.cuda.synchronize()
        outs.append((f.cpu().numpy(), back.cpu().numpy()))
    for f, back in outs[1:]:
        assert np.array_equal(f, outs[0][0])
        assert np.array_equal(back, outs[0][1])


def test_prepare_tunes_and_records_variants():
    lib = so3._lib.load()
    p = params(512, 3)
    ctx = so3.Context(0)
    ctx.prepare(p)
    got = (ctypes.c_int * 8)()
    assert lib.so3gpu_get_stage_variants(0, ctypes.byref(p.to_struct()), got) == 1
    # inverse beta / alpha and forward alpha have four 1023-point variants,
    # forward beta two; the gamma stages (length 5) only the default
    assert all(0 <= got[i] <= 3 for i in (1, 2, 5)) and 0 <= got[6] <= 1
    assert got[3] == 0 and got[4] == 0
