"""Index and sampling helpers of the drop-in C ABI (libso3gpu.so), against the
reference's known-answer tests and, exhaustively, against the checker.  Host
functions only: runs without a GPU."""
import ctypes
import itertools

import pytest

import so3_b200 as so3
from tests.helpers import oparams, params

# tests/test_sampling.c:31-143 -- (el, m, n, index)
KAT = {
    ("padded", "zero_first"): (dict(L=3, N=-1, order=0, storage=0),
                               [(0, 0, 0, 0), (2, 1, 0, 7), (2, 1, -1, 16), (2, 1, 1, 25)]),
    ("padded", "negative_first"): (dict(L=3, N=3, order=1, storage=0),
                                   [(0, 0, 0, 18), (2, -2, -2, 4), (2, 1, 0, 25), (2, 1, -1, 16), (2, 1, 1, 34)]),
    ("compact", "zero_first"): (dict(L=3, N=-1, order=0, storage=1),
                                [(0, 0, 0, 0), (2, 1, 0, 7), (2, 1, -1, 15), (2, 1, 1, 23), (2, 1, -2, 28),
                                 (2, 1, 2, 33)]),
    ("compact", "negative_first"): (dict(L=3, N=3, order=1, storage=1),
                                    [(0, 0, 0, 13), (2, -2, -2, 0), (2, 1, 0, 20), (2, 1, -1, 11), (2, 1, 1, 28),
                                     (2, 1, -2, 3), (2, 1, 2, 33)]),
}
KAT_REAL = {
    "padded": (dict(L=3, N=3, storage=0), [(0, 0, 0, 0), (2, 1, 0, 7), (2, 1, 1, 16)]),
    "compact": (dict(L=3, N=3, storage=1), [(0, 0, 0, 0), (2, 1, 0, 7), (2, 1, 1, 15), (2, 1, 2, 20)]),
}


@pytest.mark.parametrize("key", list(KAT))
def test_index_kat(key):
    kw, rows = KAT[key]
    p = params(kw["L"], kw["N"], order=kw["order"], storage=kw["storage"])
    for el, m, n, ind in rows:
        assert so3.elmn2ind(el, m, n, p) == ind
        assert so3.ind2elmn(ind, p) == (el, m, n)


@pytest.mark.parametrize("key", list(KAT_REAL))
def test_index_kat_real(key):
    kw, rows = KAT_REAL[key]
    p = params(kw["L"], kw["N"], storage=kw["storage"], reality=1)
    for el, m, n, ind in rows:
        assert so3.elmn2ind(el, m, n, p) == ind
        assert so3.ind2elmn(ind, p) == (el, m, n)


def test_convolved_parameters_kat():
    """tests/test_convolution.c:191-214."""
    f = so3.SO3Parameters(L=3, N=2, L0=1, n_order=0)
    g = so3.SO3Parameters(L=4, N=4, L0=0, n_order=0)
    h = so3.get_convolved_parameters(f, g)
    assert (h.L, h.L0, h.N) == (3, 1, 3)


@pytest.mark.parametrize("N", [8, 7, 1])
@pytest.mark.parametrize("real", [0, 1])
def test_n_loop_values(N, real):
    """tests/test_convolution.c:35-132."""
    expect = {
        0: (0, N - 1, 1) if real else (-N + 1, N - 1, 1),
        4: (0, N - 1, 1) if real else (-N + 1, N - 1, 1),
        1: (0, N - 1 if (N - 1) % 2 == 0 else N - 2, 2) if real else
        (-N + 1 if (N - 1) % 2 == 0 else -N + 2, N - 1 if (N - 1) % 2 == 0 else N - 2, 2),
        2: (1, N - 1 if (N - 1) % 2 else N - 2, 2) if real else
        (-N + 1 if (N - 1) % 2 else -N + 2, N - 1 if (N - 1) % 2 else N - 2, 2),
        3: (N - 1, N - 1, 1) if real else (-N + 1, N - 1, 2 * N - 2 if N > 1 else 1),
    }
    for mode, want in expect.items():
        assert so3.get_loop_n_values(params(8, N, reality=real, mode=mode)) == want


CASES = list(itertools.product((0, 1), (0, 1), (0, 1), (0, 1, 2, 3, 4), (1, 4, 7)))


@pytest.mark.parametrize("order,storage,real,mode,N", CASES)
def test_exhaustive_against_checker(O, order, storage, real, mode, N):
    L = 9
    p = params(L, N, L0=2, reality=real, order=order, storage=storage, mode=mode)
    op = oparams(O, p)
    lib = O.lib()
    size = so3.flmn_size(p)
    assert size == O.flmn_size(op)
    seen = set()
    for n in range(-N + 1, N):
        if real and n < 0:
            continue
        for el in range(abs(n) if storage else 0, L):
            for m in range(-el, el + 1):
                ind = so3.elmn2ind(el, m, n, p)
                want = (lib.oracle_elmn2ind_real if real else lib.oracle_elmn2ind)(el, m, n, ctypes.byref(op))
                assert ind == want
                assert 0 <= ind < size and ind not in seen
                seen.add(ind)
                assert so3.ind2elmn(ind, p) == (el, m, n)
                nz = so3.is_elmn_non_zero(el, m, n, p)
                assert nz == bool(lib.oracle_is_elmn_non_zero(el, m, n, ctypes.byref(op)))
    assert len(seen) == size


def test_sizes_and_angles():
    for sampling, steer in itertools.product((0, 1), (0, 1)):
        p = params(7, 3, sampling=sampling, steerable=steer)
        na, nb = (13, 7) if sampling == 0 else (14, 8)
        ng = 3 if steer else 5
        assert (so3.n_alpha(p), so3.n_beta(p), so3.n_gamma(p)) == (na, nb, ng)
        assert so3.f_size(p) == na * nb * ng
    lib = so3._lib.load()
    p = params(7, 3).to_struct()
    import math
    assert abs(lib.so3_sampling_b2beta(0, ctypes.byref(p)) - math.pi / 13) < 1e-15
    assert abs(lib.so3_sampling_a2alpha(2, ctypes.byref(p)) - 4 * math.pi / 13) < 1e-15
    assert abs(lib.so3_sampling_g2gamma(1, ctypes.byref(p)) - 2 * math.pi / 5) < 1e-15


def test_reference_sampling_functions_agree(O):
    """Where the reference C was built here, compare every index with it."""
    R = O.ref()
    if R is None:
        pytest.skip("reference C not built here")
    for order, storage, real in itertools.product((0, 1), (0, 1), (0, 1)):
        p = params(6, 4, reality=real, order=order, storage=storage)
        op = oparams(O, p)
        assert R.so3_sampling_flmn_size(ctypes.byref(op)) == so3.flmn_size(p)
        for i in range(so3.flmn_size(p)):
            a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            fn = R.so3_sampling_ind2elmn_real if real else R.so3_sampling_ind2elmn
            fn(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), i, ctypes.byref(op))
            assert so3.ind2elmn(i, p) == (a.value, b.value, c.value)
