"""Steerable signals (reference src/c/so3_core.c:115-126 inverse, :309-328
forward): the gamma axis is supersampled to a 2N-point circle of which the
first N samples are kept, and the forward analyses only n = N-1 (mod 2).
GPU path (through the C ABI) against the oracle's restatement and against the
reference's own C (oracle/_ref) on the same seeded inputs; 1e-12 normwise
relative error.  Real steerable transforms are rejected with status 3: the
reference's real path ignores the flag and writes 2N-1 gamma planes into a
buffer sized for N."""
import ctypes
import itertools

import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import oparams, params, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12

CASES = list(itertools.product(
    (0, 1),      # sampling MW, MWSS
    (0, 1),      # order zero-first, negative-first
    (0, 1),      # storage padded, compact
    (0, 2, 3),   # n_mode ALL, ODD, MAXIMUM
)) + [(0, 1, 0, 1), (0, 1, 0, 4)]


@pytest.mark.parametrize("sampling,order,storage,mode", CASES)
def test_steerable_against_oracle(O, sampling, order, storage, mode):
    p = params(9, 4, sampling=sampling, order=order, storage=storage, mode=mode, method=1, steerable=1)
    op = oparams(O, p)
    fl = synth.gen_flmn(p, 70 + mode)
    f = so3.inverse(fl, p)
    assert f.size == so3.f_size(p) == O.f_size(op)
    f_ref = O.inverse(fl, op)
    assert rel_err(f, f_ref) < TOL
    back = so3.forward(f_ref, p)
    assert rel_err(back, O.forward(f_ref, op)) < TOL


@pytest.mark.parametrize("L,N,sampling", [(8, 3, 0), (16, 6, 1), (64, 64, 0), (33, 5, 0)])
def test_steerable_against_reference_c(O, L, N, sampling):
    R = O.ref()
    if R is None:
        pytest.skip("reference C (oracle/_ref) not built")
    p = params(L, N, sampling=sampling, steerable=1)
    op = oparams(O, p)
    fl = synth.gen_flmn(p, L + N)
    f_ref = np.zeros(O.f_size(op), np.complex128)
    R.so3_core_inverse_via_ssht(f_ref.ctypes.data_as(ctypes.c_void_p), fl.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(op))
    assert rel_err(so3.inverse(fl, p), f_ref) < TOL
    back_ref = np.zeros(fl.size, np.complex128)
    R.so3_core_forward_via_ssht(back_ref.ctypes.data_as(ctypes.c_void_p), f_ref.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(op))
    back = so3.forward(f_ref, p)
    assert rel_err(back, back_ref) < TOL


def test_steerable_round_trip_on_its_planes():
    """A signal whose coefficients live on n = N-1 (mod 2) only comes back."""
    p = params(32, 7, steerable=1)
    fl = synth.gen_flmn(p, 5)
    for n in range(-(p.N - 1), p.N):
        if (n - (p.N - 1)) % 2:
            for el in range(abs(n), p.L):
                i0 = so3.elmn2ind(el, -el, n, p)
                fl[i0:i0 + 2 * el + 1] = 0
    assert rel_err(so3.forward(so3.inverse(fl, p), p), fl) < 1e-12


def test_steerable_device_batch_matches_single():
    import torch
    p = params(24, 5, steerable=1)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 40 + i)).cuda() for i in range(3)]
    one = [ctx.inverse(x, p) for x in fls]
    mx = ctx.inverse_batch(fls, p, "mixed")
    torch.cuda.synchronize()
    for a, b in zip(mx, one):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-10
    back = ctx.forward_batch(one, p, "mixed")
    ref = [ctx.forward(x, p) for x in one]
    torch.cuda.synchronize()
    for a, b in zip(back, ref):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-10


def test_steerable_real_is_rejected():
    p = params(8, 4, reality=1, steerable=1)
    with pytest.raises(so3.SO3Error, match="status 3"):
        so3.inverse(np.zeros(so3.flmn_size(p), complex), p)
