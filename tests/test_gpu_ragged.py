"""Ragged split-precision batches: signals of different parameters (L, N, L0,
sampling, storage, n-order, n-mode, recursion) in one call, their Wigner
contractions in one tensor-core launch per recursion (groups of 16 similar
signals at the group's largest L and N).  Each result against the same
signal's FP64 transform: <= 1e-10 normwise relative error (the split path's
contract); the FP64 form of the ragged call equals the single calls exactly."""
import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import params, rel_err

pytestmark = pytest.mark.gpu


def _mix():
    ps = [params(40, 7), params(16, 16), params(33, 5, sampling=1, method=1), params(64, 3, L0=5),
          params(24, 9, order=0, storage=1), params(20, 6, mode=1), params(20, 6, mode=3), params(1, 1),
          params(70, 2), params(8, 8, reality=1), params(30, 4, steerable=1), params(48, 12, method=1)]
    rng = np.random.default_rng(3)
    for i in range(10):  # a second group of similar sizes
        ps.append(params(int(rng.integers(8, 40)), int(rng.integers(1, 8))))
    return ps


def test_ragged_split_matches_fp64_per_signal(monkeypatch):
    import torch
    ctx = so3.Context(0)
    ps = _mix()
    fls = [torch.from_numpy(synth.gen_flmn(p, 60 + i)).cuda() for i, p in enumerate(ps)]
    one = [ctx.inverse(x, p) for x, p in zip(fls, ps)]
    mx = ctx.inverse_ragged(fls, ps, "mixed")
    torch.cuda.synchronize()
    assert so3.take_kernel_error() == 0
    for a, b, p in zip(mx, one, ps):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) <= 1e-10, p
    back1 = [ctx.forward(x, p) for x, p in zip(one, ps)]
    backm = ctx.forward_ragged(one, ps, "mixed")
    torch.cuda.synchronize()
    assert so3.take_kernel_error() == 0
    for a, b, p in zip(backm, back1, ps):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) <= 1e-10, p


def test_ragged_fp64_equals_single_calls():
    import torch
    ctx = so3.Context(0)
    ps = _mix()[:8]
    fls = [torch.from_numpy(synth.gen_flmn(p, 80 + i)).cuda() for i, p in enumerate(ps)]
    one = [ctx.inverse(x, p) for x, p in zip(fls, ps)]
    rag = ctx.inverse_ragged(fls, ps, "fp64")
    torch.cuda.synchronize()
    for a, b in zip(rag, one):
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())


def test_ragged_uniform_batch_matches_batch_call():
    """One geometry through the ragged path equals the uniform split batch
    within the split tolerance (the same digits and products, different
    kernels)."""
    import torch
    ctx = so3.Context(0)
    p = params(48, 6)
    fls = [torch.from_numpy(synth.gen_flmn(p, 90 + i)).cuda() for i in range(5)]
    a = ctx.inverse_batch(fls, p, "mixed")
    b = ctx.inverse_ragged(fls, [p] * 5, "mixed")
    c = ctx.inverse_batch(fls, p, "fp64")
    torch.cuda.synchronize()
    for x, y, z in zip(a, b, c):
        assert rel_err(y.cpu().numpy(), z.cpu().numpy()) <= 1e-10
        assert rel_err(x.cpu().numpy(), y.cpu().numpy()) <= 1e-10


def test_ragged_with_small_delta_table_in_fresh_process():
    """A ragged split call in a fresh process whose signals need only a small
    Delta(pi/2) table: no covering digit table exists, and none may be built
    from a Delta table that does not hold the planes up to l = 511 (the
    products then generate A from Delta).  Run in a child process so that no
    table of an earlier test is resident."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import torch, so3_b200 as so3\n"
        "from so3_b200 import synth\n"
        "from tests.helpers import params, rel_err\n"
        "ps = [params(20, 4, method=1), params(33, 6, method=1), params(40, 3, method=1), params(24, 5)]\n"
        "ctx = so3.Context(0)\n"
        "fls = [torch.from_numpy(synth.gen_flmn(p, 5 + i)).cuda() for i, p in enumerate(ps)]\n"
        "one = [ctx.inverse(x, p) for x, p in zip(fls, ps)]\n"
        "mx = ctx.inverse_ragged(fls, ps, 'mixed')\n"
        "bk = ctx.forward_ragged(one, ps, 'mixed')\n"
        "torch.cuda.synchronize()\n"
        "assert so3.take_kernel_error() == 0\n"
        "for a, b in zip(mx, one): assert rel_err(a.cpu().numpy(), b.cpu().numpy()) <= 1e-10\n"
        "for a, x in zip(bk, fls): assert rel_err(a.cpu().numpy(), x.cpu().numpy()) <= 1e-10\n"
        "print('ok')\n" % root)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]
