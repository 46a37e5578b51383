"""The CPU checker itself: pinned against closed forms, the reference's own
self-consistency tests and (where it was built here) the reference C.

Runs without a GPU."""
import itertools
from math import cos, factorial, pi, sin, sqrt

import numpy as np
import pytest

from so3_b200 import synth
from tests.helpers import params, oparams, rel_err


def wigner_d(j, mp, m, beta):
    """Wigner's explicit sum (standard Condon-Shortley convention)."""
    c, s = cos(beta / 2), sin(beta / 2)
    pre = sqrt(factorial(j + mp) * factorial(j - mp) * factorial(j + m) * factorial(j - m))
    tot = 0.0
    for k in range(0, 2 * j + 1):
        if j + m - k < 0 or mp - m + k < 0 or j - mp - k < 0:
            continue
        tot += (-1) ** (mp - m + k) * c ** (2 * j + m - mp - 2 * k) * s ** (mp - m + 2 * k) / (
            factorial(j + m - k) * factorial(k) * factorial(mp - m + k) * factorial(j - mp - k))
    return pre * tot


@pytest.mark.parametrize("method", [0, 1])
def test_delta_planes_match_wigner_formula(O, method):
    worst = 0.0
    for el in range(0, 9):
        D = O.dl_plane(12, el, method)
        for a in range(el + 1):
            for b in range(el + 1):
                worst = max(worst, abs(D[a, b] - wigner_d(el, a, b, pi / 2)))
    assert worst < 1e-14


def test_risbo_and_trapani_agree_and_are_orthogonal(O):
    l = 300
    R = O.dl_plane(400, l, 0)
    T = O.dl_plane(400, l, 1)
    assert np.abs(R - T).max() < 1e-13
    # full matrix from the quarter by Delta_{-m',m} = (-1)^{l+m} Delta_{m'm}, Delta_{m',-m} = (-1)^{l+m'} ...
    idx = np.arange(-l, l + 1)
    F = R[np.abs(idx)[:, None], np.abs(idx)[None, :]].copy()
    sgn = np.ones_like(F)
    sgn *= np.where(idx[:, None] < 0, (-1.0) ** (l + np.abs(idx)[None, :]), 1.0)
    sgn *= np.where(idx[None, :] < 0, (-1.0) ** (l + np.abs(idx)[:, None]), 1.0)
    F *= sgn
    assert np.abs(F @ F.T - np.eye(2 * l + 1)).max() < 1e-12


def _naive_inverse(flmn, p, O):
    L, N = p.L, p.N
    mw = p.sampling_scheme == 0
    na, nb, ng = (2 * L - 1, L, 2 * N - 1) if mw else (2 * L, L + 1, 2 * N - 1)
    al = 2 * pi * np.arange(na) / na
    be = (2 * np.arange(nb) + 1) * pi / (2 * L - 1) if mw else np.arange(nb) * pi / L
    ga = 2 * pi * np.arange(ng) / ng
    f = np.zeros((ng, nb, na), complex)
    for n in range(-N + 1, N):
        for el in range(abs(n), L):
            for m in range(-el, el + 1):
                c = flmn[synth.block_base(p, n) + el * el + el + m]
                if c == 0:
                    continue
                d = np.array([wigner_d(el, m, n, b) for b in be])
                f += (2 * el + 1) / (8 * pi ** 2) * c * np.exp(1j * n * ga)[:, None, None] * d[None, :, None] \
                    * np.exp(1j * m * al)[None, None, :]
    return f.ravel()


@pytest.mark.parametrize("sampling", [0, 1])
def test_inverse_matches_closed_form(O, sampling):
    """f(a,b,g) = sum (2l+1)/(8 pi^2) f_lmn e^{i m alpha} d^l_mn(beta) e^{i n gamma}."""
    p = params(5, 3, sampling=sampling)
    fl = synth.gen_flmn(p, 1)
    assert rel_err(O.inverse(fl, oparams(O, p)), _naive_inverse(fl, p, O)) < 1e-13


ROUND_TRIP = list(itertools.product((0, 1), (0, 1), (0, 1), (0, 1, 2, 3, 4), (0, 1)))


@pytest.mark.parametrize("sampling,order,storage,mode,real", ROUND_TRIP)
def test_round_trip_matrix(O, sampling, order, storage, mode, real):
    """The reference's test_back_and_forth matrix (tests/test_so3.c:98-133,
    :255-326) at L=8, N=8, Trapani -- here with 1e-12 instead of 1e-8."""
    p = params(8, 8, reality=real, sampling=sampling, order=order, storage=storage, mode=mode, method=1)
    op = oparams(O, p)
    fl = synth.gen_flmn(p, 10)
    back = O.forward(O.inverse(fl, op), op)
    assert rel_err(back, fl) < 1e-12


def _ref_or_skip(O):
    R = O.ref()
    if R is None:
        pytest.skip("reference C not built here (oracle/_ref)")
    return R


@pytest.mark.parametrize("sampling,order,storage,mode,real", ROUND_TRIP)
def test_oracle_equals_reference_c(O, sampling, order, storage, mode, real):
    """Restatement vs the reference's own so3_core.c compiled against the same
    stand-ins: identical algorithm, so agreement to rounding."""
    _ref_or_skip(O)
    p = params(9, 4, L0=1, reality=real, sampling=sampling, order=order, storage=storage, mode=mode)
    op = oparams(O, p)
    fl = synth.gen_flmn(p, 3)
    f = O.inverse(fl, op)
    assert rel_err(f, O.ref_inverse(fl, op)) < 1e-14
    assert rel_err(O.forward(f, op), O.ref_forward(f, op)) < 1e-14


@pytest.mark.parametrize("real", [0, 1])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_reference_direct_equals_via_ssht(O, real, mode):
    """The reference's test_direct_vs_ssht (tests/test_so3.c:135-188): its
    in-tree direct transform (ssht_dl_* + FFTW only) against the via-SSHT
    transform that runs the SSHT stand-in.  Pins the spin transforms to the
    algorithm the reference states in its own source."""
    _ref_or_skip(O)
    p = params(8, 8, reality=real, mode=mode, method=1)
    op = oparams(O, p)
    fl = synth.gen_flmn(p, 10)
    assert rel_err(O.ref_inverse(fl, op, direct=True), O.ref_inverse(fl, op)) < 1e-13
    # forward on arbitrary (not band-limited) samples: the quadrature itself
    rng = np.random.default_rng(4)
    n = O.f_size(op)
    f = rng.normal(size=n) if real else rng.normal(size=n) + 1j * rng.normal(size=n)
    assert rel_err(O.ref_forward(f, op, direct=True), O.ref_forward(f, op)) < 1e-13


def test_golden_fixtures(O):
    """Oracle reproduces the committed fixtures generated from the reference C."""
    import glob
    import json
    import os
    files = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
    assert files, "no golden fixtures committed"
    for fn in files:
        z = np.load(fn)
        cfg = json.loads(str(z["config"]))
        op = O.params(**cfg)
        f = O.inverse(z["flmn"], op)
        assert rel_err(f, z["f"]) < 1e-13, fn
        assert rel_err(O.forward(z["f"], op), z["flmn_back"]) < 1e-13, fn


def test_harmonic_convolution_oracle_matches_reference(O):
    R = _ref_or_skip(O)
    import ctypes
    for real in (0, 1):
        for N in (8, 7, 1):
            p = params(8, N, reality=real)
            op = oparams(O, p)
            f = synth.gen_flmn(p, 1)
            g = synth.gen_flmn(p, 2)
            h, hp = O.harmonic_convolution(f, op, g, op)
            hr = np.zeros_like(h)
            R.so3_conv_harmonic_convolution(hr.ctypes.data_as(ctypes.c_void_p), ctypes.byref(hp),
                                            f.ctypes.data_as(ctypes.c_void_p), ctypes.byref(op),
                                            g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(op))
            assert np.abs(h - hr).max() < 1e-12


def test_reference_adjoints_are_adjoint_to_its_direct_transforms(O):
    """Pins the reference's adjoint build (src/c/so3_adjoint.c) against its own
    direct transforms: <y, A x> = <A^H y, x> for the inverse and forward."""
    import numpy as np
    from so3_b200 import synth
    from tests.helpers import oparams, params
    if O.ref() is None:
        import pytest
        pytest.skip("reference C (oracle/_ref) not built")
    for p in (params(8, 4), params(6, 6, mode=2, L0=2), params(7, 3, storage=1, order=0, method=1)):
        op = oparams(O, p)
        rng = np.random.default_rng(1)
        x = synth.gen_flmn(p, 3)
        y = rng.normal(size=O.f_size(op)) + 1j * rng.normal(size=O.f_size(op))
        a = np.vdot(y, O.ref_inverse(x, op, direct=True))
        assert abs(a - np.vdot(O.ref_adjoint_inverse(y, op), x)) / abs(a) < 1e-13
        z = synth.gen_flmn(p, 5)
        b = np.vdot(z, O.ref_forward(y, op, direct=True))
        assert abs(b - np.vdot(O.ref_adjoint_forward(z, op), y)) / abs(b) < 1e-13
