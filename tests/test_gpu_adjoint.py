"""Adjoint transforms (reference src/c/so3_adjoint.c:34 so3_adjoint_inverse_direct,
:402 so3_adjoint_forward_direct, :939 / :1313 their _real variants; MW) through
the drop-in C ABI:

* against the reference's own C (oracle/_ref, compiled unmodified) on the
  same seeded inputs, 1e-12 normwise relative error;
* the defining identity <y, A x> = <A^H y, x> with the GPU's own inverse and
  forward transforms at sizes the CPU would take long for (size-independent
  property)."""
import itertools

import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import oparams, params, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12

CASES = list(itertools.product((0, 1), (0, 1), (0, 1, 2, 3), (0, 1))) + [(1, 0, 0, 0)]


@pytest.mark.parametrize("order,storage,mode,method", CASES)
def test_adjoints_against_reference_c(O, order, storage, mode, method):
    if O.ref() is None:
        pytest.skip("reference C (oracle/_ref) not built")
    p = params(9, 5, L0=1 if mode == 0 else 0, order=order, storage=storage, mode=mode, method=method)
    op = oparams(O, p)
    rng = np.random.default_rng(17 + mode)
    f = rng.normal(size=O.f_size(op)) + 1j * rng.normal(size=O.f_size(op))
    assert rel_err(so3.adjoint_inverse(f, p), O.ref_adjoint_inverse(f, op)) < TOL
    fl = synth.gen_flmn(p, 23 + mode)
    assert rel_err(so3.adjoint_forward(fl, p), O.ref_adjoint_forward(fl, op)) < TOL


@pytest.mark.parametrize("L,N", [(1, 1), (2, 2), (16, 1), (33, 7)])
def test_adjoint_edge_sizes_against_reference_c(O, L, N):
    if O.ref() is None:
        pytest.skip("reference C (oracle/_ref) not built")
    p = params(L, N)
    op = oparams(O, p)
    rng = np.random.default_rng(L + N)
    f = rng.normal(size=O.f_size(op)) + 1j * rng.normal(size=O.f_size(op))
    assert rel_err(so3.adjoint_inverse(f, p), O.ref_adjoint_inverse(f, op)) < TOL
    fl = synth.gen_flmn(p, 5)
    assert rel_err(so3.adjoint_forward(fl, p), O.ref_adjoint_forward(fl, op)) < TOL


@pytest.mark.parametrize("order,storage,mode,method", CASES)
def test_real_adjoints_against_reference_c(O, order, storage, mode, method):
    if O.ref() is None:
        pytest.skip("reference C (oracle/_ref) not built")
    p = params(9, 5, L0=1 if mode == 0 else 0, reality=1, order=order, storage=storage, mode=mode,
               method=method)
    op = oparams(O, p)
    rng = np.random.default_rng(31 + mode)
    f = rng.normal(size=O.f_size(op))
    assert rel_err(so3.adjoint_inverse(f, p), O.ref_adjoint_inverse_real(f, op)) < TOL
    fl = rng.normal(size=so3.flmn_size(p)) + 1j * rng.normal(size=so3.flmn_size(p))
    assert rel_err(so3.adjoint_forward(fl, p), O.ref_adjoint_forward_real(fl, op)) < TOL


@pytest.mark.parametrize("L,N", [(1, 1), (2, 2), (16, 1), (33, 7), (64, 16)])
def test_real_adjoint_edge_sizes_against_reference_c(O, L, N):
    if O.ref() is None:
        pytest.skip("reference C (oracle/_ref) not built")
    p = params(L, N, reality=1)
    op = oparams(O, p)
    rng = np.random.default_rng(3 * L + N)
    f = rng.normal(size=O.f_size(op))
    assert rel_err(so3.adjoint_inverse(f, p), O.ref_adjoint_inverse_real(f, op)) < TOL
    fl = rng.normal(size=so3.flmn_size(p)) + 1j * rng.normal(size=so3.flmn_size(p))
    assert rel_err(so3.adjoint_forward(fl, p), O.ref_adjoint_forward_real(fl, op)) < TOL


@pytest.mark.parametrize("L,N", [(64, 64), (128, 8)])
def test_adjoint_identity_with_gpu_transforms(L, N):
    p = params(L, N)
    rng = np.random.default_rng(L)
    x = synth.gen_flmn(p, 1)
    y = rng.normal(size=so3.f_size(p)) + 1j * rng.normal(size=so3.f_size(p))
    lhs = np.vdot(y, so3.inverse(x, p))
    rhs = np.vdot(so3.adjoint_inverse(y, p), x)
    assert abs(lhs - rhs) / abs(lhs) < 1e-12
    z = synth.gen_flmn(p, 2)
    lhs = np.vdot(z, so3.forward(y, p))
    rhs = np.vdot(so3.adjoint_forward(z, p), y)
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


@pytest.mark.parametrize("kw", [dict(sampling=1), dict(sampling=1, reality=1), dict(steerable=1)])
def test_adjoint_rejects_unsupported(kw):
    p = params(8, 4, **kw)
    with pytest.raises(so3.SO3Error, match="status 3"):
        so3.adjoint_forward(np.zeros(so3.flmn_size(p), complex), p)
