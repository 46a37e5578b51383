"""Drop-in calls on host buffers run as a pipeline: the coefficient blocks
(grouped by |n|) and the sample rows (grouped by beta) are copied in chunks
that overlap the kernels of the other chunks.  With the chunk threshold
lowered to one byte every call below is chunked; results must equal the
oracle within the parity tolerance and the unchunked device-pointer path
exactly (same kernels, same per-CTA arithmetic)."""
import ctypes

import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import oparams, params, rel_err

TOL = 1e-12

pytestmark = pytest.mark.gpu


@pytest.fixture
def chunked(monkeypatch):
    monkeypatch.setenv("SO3GPU_STAGE_CHUNK_BYTES", "1")


CASES = [
    dict(L=24, N=9),
    dict(L=24, N=9, order=0, storage=1),
    dict(L=20, N=7, sampling=1, storage=1, method=1),
    dict(L=24, N=9, reality=1),
    dict(L=22, N=8, reality=1, sampling=1, storage=1),
    dict(L=24, N=9, mode=1),
    dict(L=24, N=9, mode=3, order=0),
    dict(L=18, N=1, reality=1),
    dict(L=24, N=2, L0=3),
]


@pytest.mark.parametrize("kw", CASES, ids=[str(i) for i in range(len(CASES))])
def test_chunked_dropin_matches_oracle_and_device_path(O, chunked, kw):
    import torch
    kw = dict(kw)
    L, N = kw.pop("L"), kw.pop("N")
    p = params(L, N, **kw)
    op = oparams(O, p)
    fl = synth.gen_flmn(p, 11)
    f_host = so3.inverse(fl, p)
    f_ref = O.inverse(fl, op)
    assert rel_err(f_host, f_ref) < TOL
    ctx = so3.Context(0)
    f_dev = ctx.inverse(torch.from_numpy(fl).cuda(), p)
    torch.cuda.synchronize()
    assert np.array_equal(f_dev.cpu().numpy(), f_host)
    back = so3.forward(f_ref, p)
    assert rel_err(back, O.forward(f_ref, op)) < TOL
    back_dev = ctx.forward(torch.from_numpy(np.ascontiguousarray(f_ref)).cuda(), p)
    torch.cuda.synchronize()
    if p.n_mode == 0:
        assert np.array_equal(back_dev.cpu().numpy(), back)


def test_chunked_forward_keeps_skipped_blocks(O, chunked):
    p = params(24, 9, mode=1)
    fl = synth.gen_flmn(p, 3)
    f = O.inverse(fl, oparams(O, p))
    out = np.full(so3.flmn_size(p), 7.0 + 1j)
    lib = so3._lib.load()
    lib.so3_core_forward_via_ssht(out.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p),
                                  ctypes.byref(p.to_struct()))
    so3._lib.check()
    ref = np.full(so3.flmn_size(p), 7.0 + 1j)
    O.forward(f, oparams(O, p), out=ref)
    assert rel_err(out, ref) < TOL


def test_chunked_direct_forward_zeroes_skipped_blocks(O, chunked):
    p = params(24, 9, mode=2)
    fl = synth.gen_flmn(p, 5)
    f = O.inverse(fl, oparams(O, p))
    out = np.full(so3.flmn_size(p), 7.0 + 1j)
    lib = so3._lib.load()
    lib.so3_core_forward_direct(out.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(p.to_struct()))
    so3._lib.check()
    ref = np.zeros(so3.flmn_size(p), complex)
    O.forward(f, oparams(O, p), out=ref)
    assert rel_err(out, ref) < TOL


def test_chunked_pinned_buffers_round_trip(chunked):
    """Page-locked host buffers (asynchronous copies) through the same entry points."""
    import torch
    p = params(32, 12)
    fl = torch.from_numpy(synth.gen_flmn(p, 2)).pin_memory()
    f = torch.empty(so3.f_size(p), dtype=torch.complex128).pin_memory()
    back = torch.empty_like(fl).pin_memory()
    lib = so3._lib.load()
    q = p.to_struct()
    for _ in range(2):
        lib.so3_core_inverse_via_ssht(ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(fl.data_ptr()), ctypes.byref(q))
        lib.so3_core_forward_via_ssht(ctypes.c_void_p(back.data_ptr()), ctypes.c_void_p(f.data_ptr()),
                                      ctypes.byref(q))
        so3._lib.check()
        assert rel_err(back.numpy(), fl.numpy()) < 1e-11
