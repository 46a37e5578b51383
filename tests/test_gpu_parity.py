"""GPU parity: the sm_100a path (through the C ABI) against the CPU oracle on
the same seeded inputs.  Tolerance: 1e-12 normwise relative error (max |x-y| /
max |y|) for every transform, as the transform-path contract states."""
import itertools

import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import oparams, params, rel_err

TOL = 1e-12

pytestmark = pytest.mark.gpu


def _both(O, p, seed=7, dist="uniform"):
    fl = synth.gen_flmn(p, seed, dist)
    op = oparams(O, p)
    f_gpu = so3.inverse(fl, p)
    f_ref = O.inverse(fl, op)
    return fl, op, f_gpu, f_ref


MATRIX = list(itertools.product(
    (0, 1),        # sampling MW, MWSS
    (0, 1),        # order zero-first, negative-first
    (0, 1),        # storage padded, compact
    (0, 1, 2, 3, 4),  # n_mode
    (0, 1),        # Risbo, Trapani
    (0, 1),        # complex, real
))


@pytest.mark.parametrize("sampling,order,storage,mode,method,real", MATRIX)
def test_small_matrix(O, sampling, order, storage, mode, method, real):
    p = params(8, 5, L0=1, reality=real, sampling=sampling, order=order, storage=storage, mode=mode,
               method=method)
    fl, op, f_gpu, f_ref = _both(O, p)
    assert rel_err(f_gpu, f_ref) < TOL
    # forward on the GPU and on the oracle from the same samples (both start
    # from zeroed coefficients, so skipped n-blocks compare as zero)
    fl_g = so3.forward(f_ref, p)
    fl_o = O.forward(f_ref, op)
    assert rel_err(fl_g, fl_o) < TOL
    assert rel_err(fl_g, fl) < 1e-11  # round trip


@pytest.mark.parametrize("L,N,L0", [(1, 1, 0), (2, 1, 0), (2, 2, 0), (3, 2, 1), (4, 4, 3), (7, 7, 0), (16, 1, 0),
                                    (16, 8, 0), (16, 8, 1), (17, 3, 5)])
@pytest.mark.parametrize("real", [0, 1])
@pytest.mark.parametrize("sampling", [0, 1])
def test_edge_sizes(O, L, N, L0, real, sampling):
    p = params(L, N, L0=L0, reality=real, sampling=sampling)
    fl, op, f_gpu, f_ref = _both(O, p, seed=L * 31 + N)
    assert rel_err(f_gpu, f_ref) < TOL
    fl_g = so3.forward(f_ref, p)
    assert rel_err(fl_g, O.forward(f_ref, op)) < TOL


@pytest.mark.parametrize("N", [1, 2])
def test_metric_lengths_L512_against_oracle(O, N):
    """L=512 runs the compile-time DFT plans (1023 = 31*11*3 over alpha and the
    extended beta circle, 2048 for the weight convolution); compared with the
    oracle on a few n-planes, inverse and forward (forward on the oracle's
    samples)."""
    p = params(512, N)
    fl, op, f_gpu, f_ref = _both(O, p, seed=512 + N)
    assert rel_err(f_gpu, f_ref) < TOL
    assert rel_err(so3.forward(f_ref, p), O.forward(f_ref, op)) < TOL


def test_config_complex_L64_N64_risbo(O):
    """Plain complex round trip, MW, L=64, N=64, padded, all n, Risbo, U(-1,1)."""
    p = params(64, 64)
    fl, op, f_gpu, f_ref = _both(O, p, seed=2024)
    assert rel_err(f_gpu, f_ref) < TOL
    fl_g = so3.forward(f_gpu, p)
    fl_o = O.forward(f_ref, op)
    assert rel_err(fl_g, fl_o) < TOL
    assert rel_err(fl_g, fl) < 1e-11


def test_config_real_mwss_L256_N32_trapani(O):
    """Real signal, MWSS, L=256, N=32, compact, Trapani, Gaussian (l+1)^-2."""
    p = params(256, 32, reality=1, sampling=1, storage=1, method=1)
    fl, op, f_gpu, f_ref = _both(O, p, seed=11, dist="gauss")
    assert rel_err(f_gpu, f_ref) < TOL
    fl_g = so3.forward(f_gpu, p)
    fl_o = O.forward(f_ref, op)
    assert rel_err(fl_g, fl_o) < TOL
    assert rel_err(fl_g, fl) < 1e-11


@pytest.mark.parametrize("L,N", [(128, 16), (512, 4)])
def test_round_trip_large(L, N):
    """Size-independent property at larger L: forward(inverse(flmn)) == flmn."""
    p = params(L, N)
    fl = synth.gen_flmn(p, 5, "gauss")
    f = so3.inverse(fl, p)
    assert rel_err(so3.forward(f, p), fl) < 1e-11


def test_forward_leaves_skipped_blocks(O):
    """n_mode != ALL: blocks of skipped n keep the caller's contents."""
    import ctypes
    p = params(8, 4, mode=1)
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


def test_direct_entry_points_match(O):
    p = params(12, 6)
    fl = synth.gen_flmn(p, 9)
    import ctypes
    lib = so3._lib.load()
    f = np.zeros(so3.f_size(p), complex)
    lib.so3_core_inverse_direct(f.ctypes.data_as(ctypes.c_void_p), fl.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(p.to_struct()))
    so3._lib.check()
    assert rel_err(f, O.inverse(fl, oparams(O, p))) < TOL


def test_s2toso3(O):
    L, N = 32, 8
    hp = params(L, N)
    flm = synth.gen_flm(L, 1)
    glm = synth.gen_flm(L, 2, mmax=N - 1)
    h = so3.s2toso3_harmonic_convolution(hp, flm, glm)
    assert rel_err(h, O.s2toso3(oparams(O, hp), flm, glm)) < TOL


@pytest.mark.parametrize("real", [0, 1])
@pytest.mark.parametrize("N", [8, 7, 1])
def test_harmonic_convolution(O, real, N):
    p = params(8, N, reality=real)
    f = synth.gen_flmn(p, 1)
    g = synth.gen_flmn(p, 2)
    h, hp = so3.convolve_harmonic(f, p, g, p)
    ho, hpo = O.harmonic_convolution(f, oparams(O, p), g, oparams(O, p))
    assert (hp.L, hp.N, hp.L0) == (hpo.L, hpo.N, hpo.L0)
    assert rel_err(h, ho) < TOL


def test_invalid_parameters_return_status():
    p = params(8, 4)
    p.sampling_scheme = 7
    with pytest.raises(so3.SO3Error, match="status 1"):
        so3.inverse(np.zeros(8 * 8 * 7, complex), p)
    p = params(8, 4, mode=9)
    with pytest.raises(so3.SO3Error, match="status 1"):
        so3.inverse(np.zeros(8 * 8 * 7, complex), p)
    p = params(8, 4, steerable=1, reality=1)  # steerable: complex transforms only
    with pytest.raises(so3.SO3Error, match="status 3"):
        so3.inverse(np.zeros(8 * 8 * 4, complex), p)


def test_device_api_matches_host_api():
    import torch
    p = params(32, 8)
    fl = synth.gen_flmn(p, 4)
    ctx = so3.Context(0)
    ctx.prepare(p)
    f_dev = ctx.inverse(torch.from_numpy(fl).cuda(), p)
    torch.cuda.synchronize()
    f_host = so3.inverse(fl, p)
    assert rel_err(f_dev.cpu().numpy(), f_host) < 1e-15
    back = ctx.forward(f_dev, p)
    torch.cuda.synchronize()
    assert rel_err(back.cpu().numpy(), fl) < 1e-11


@pytest.mark.parametrize("Lf,Lg", [(8, 8), (10, 7)])
def test_real_space_convolution_against_reference(O, Lf, Lg):
    """so3_conv_convolution (reference src/c/so3_conv.c:154-184: forward of f
    and g, harmonic convolution, inverse into h's samples) through the C ABI,
    against the reference's own C in oracle/_ref on the same samples."""
    import ctypes
    R = O.ref()
    if R is None:
        pytest.skip("reference C (oracle/_ref) not built")
    fp, gp = params(Lf, Lf), params(Lg, Lg)
    f = O.inverse(synth.gen_flmn(fp, 31), oparams(O, fp))
    g = O.inverse(synth.gen_flmn(gp, 32), oparams(O, gp))
    h, hp = so3.convolve(f, fp, g, gp)
    assert (hp.L, hp.N) == (min(Lf, Lg), min(Lf, Lg))
    hop = oparams(O, hp)
    h_ref = np.zeros(O.f_size(hop), np.complex128)
    R.so3_conv_convolution(h_ref.ctypes.data_as(ctypes.c_void_p), ctypes.byref(hop),
                           f.ctypes.data_as(ctypes.c_void_p), ctypes.byref(oparams(O, fp)),
                           g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(oparams(O, gp)))
    assert rel_err(h, h_ref) < TOL
