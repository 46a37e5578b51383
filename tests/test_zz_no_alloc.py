"""so3gpu_inverse_noalloc -- the inverse transform for callers that cannot call
cudaMalloc: code running under an allocator or memory cap owned by someone
else, or loops that must not allocate after start-up.  Its scratch and tables
are static device arrays; its results must equal the allocating entry
point's, and a call after the first must leave the device's free memory
unchanged.

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


# (parameters, seed): the 127-point DFTs (MW L=64 over alpha and the extended beta
# circle, N=64 over gamma) run the fixed Bluestein engine on this entry point's
# own tables; L=62 (P=123) the generic Bluestein engine; L=64, N=64 is the
# documented maximum (33.2 MB of the 32 MiB = 33.55 MB scratch array)
CASES = [
    (so3.SO3Parameters(L=32, N=8), 1),
    (so3.SO3Parameters(L=32, N=8), 2),  # second call in a row, same band limits
    (so3.SO3Parameters(L=16, N=5, sampling_scheme=1, storage=1, dl_method=1), 3),  # tables change
    (so3.SO3Parameters(L=32, N=64), 4),
    (so3.SO3Parameters(L=62, N=9, dl_method=1), 5),
    (so3.SO3Parameters(L=64, N=64), 6),
    (so3.SO3Parameters(L=64, N=64, sampling_scheme=1, n_order=0), 7),
]


def test_noalloc_matches_allocating_entry_point():
    import torch
    lib = so3._lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    ctx = so3.Context(0, stream=torch.cuda.current_stream())
    for p, seed in CASES:
        fl = torch.from_numpy(synth.gen_flmn(p, seed)).cuda()
        ref = ctx.inverse(fl, p)
        for rep in range(2):  # two calls in a row on the same input
            out = torch.full_like(ref, complex(np.nan, np.nan))
            assert _noalloc(lib, out, fl, p, stream) == 0, lib.so3gpu_last_error()
            torch.cuda.synchronize()
            err = float(((out - ref).abs().max() / ref.abs().max()).item())
            assert err < TOL, (p, rep, err)


def test_noalloc_allocates_nothing_after_the_first_call():
    import torch
    lib = so3._lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    p = so3.SO3Parameters(L=64, N=64)
    fl = torch.from_numpy(synth.gen_flmn(p, 11)).cuda()
    out = torch.empty(so3.f_size(p), dtype=torch.complex128, device="cuda")
    assert _noalloc(lib, out, fl, p, stream) == 0, lib.so3gpu_last_error()  # set-up, kernels loaded
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _noalloc(lib, out, fl, p, stream) == 0, lib.so3gpu_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_what_its_arrays_cannot_hold():
    """Rejected on the host before any device work (status 3): band limits
    beyond the arrays, real signals (their buffers are sized for the real
    layout) and steerable signals.  The buffers are sized for the complex
    layout of each request, so nothing is read or written out of bounds even
    if a check were missing."""
    import torch
    lib = so3._lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for kw in (dict(L=128, N=8), dict(L=65, N=4), dict(L=16, N=65), dict(L=16, N=4, reality=1),
               dict(L=16, N=4, steerable=1)):
        p = so3.SO3Parameters(**kw)
        pc = so3.SO3Parameters(**dict(kw, reality=0, steerable=0))
        fl = torch.zeros(so3.flmn_size(pc), dtype=torch.complex128, device="cuda")
        out = torch.zeros(so3.f_size(pc), dtype=torch.complex128, device="cuda")
        assert _noalloc(lib, out, fl, p, stream) == 3, kw
        msg = lib.so3gpu_last_error()
        assert b"noalloc" in msg, (kw, msg)
