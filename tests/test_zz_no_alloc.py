"""so3gpu_inverse_noalloc -- the inverse transform for callers that cannot call
cudaMalloc (code under a foreign allocator or memory cap, or loops that must
not allocate after start-up).  Its scratch and tables are static device
arrays; its results must equal the allocating entry point's.

Collected last on purpose: a run that stops at the first failure has already
run every other test.  Passes alone in a fresh process and after the others.
"""
import ctypes

import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-12  # normwise relative error, as in the other parity tests


def _noalloc(lib, out, flmn, p, stream):
    return lib.so3gpu_inverse_noalloc(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(flmn.data_ptr()),
                                      ctypes.byref(p.to_struct()), ctypes.c_void_p(stream))


def test_noalloc_matches_allocating_entry_point():
    import torch
    lib = so3._lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    ctx = so3.Context(0, stream=torch.cuda.current_stream())
    cases = [
        (so3.SO3Parameters(L=32, N=8), 1),
        (so3.SO3Parameters(L=32, N=8), 2),  # second call in a row, same band limits
        (so3.SO3Parameters(L=16, N=5, sampling_scheme=1, storage=1, dl_method=1), 3),  # tables change
    ]
    for p, seed in cases:
        fl = torch.from_numpy(synth.gen_flmn(p, seed)).cuda()
        ref = ctx.inverse(fl, p)
        out = torch.full_like(ref, complex(np.nan, np.nan))
        assert _noalloc(lib, out, fl, p, stream) == 0, lib.so3gpu_last_error()
        torch.cuda.synchronize()
        err = float(((out - ref).abs().max() / ref.abs().max()).item())
        assert err < TOL, (p, err)


def test_noalloc_rejects_sizes_beyond_its_arrays():
    import torch
    lib = so3._lib.load()
    p = so3.SO3Parameters(L=128, N=8)
    fl = torch.zeros(so3.flmn_size(p), dtype=torch.complex128, device="cuda")
    out = torch.zeros(so3.f_size(p), dtype=torch.complex128, device="cuda")
    assert _noalloc(lib, out, fl, p, torch.cuda.current_stream().cuda_stream) == 3
    assert b"noalloc" in lib.so3gpu_last_error()
