"""ctypes front end of the CPU checker libraries.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline leg; the GPU product never imports it.

Two libraries are wrapped:

* ``oracle/lib/liboracle.so`` -- the project's C restatement of the SO3
  reference's via-SSHT transform path (``so3_oracle.c``) plus the project's
  SSHT and FFTW stand-ins.  Always buildable (``make -C oracle lib``).
* ``oracle/_ref/libso3ref.so`` -- the reference's own ``src/c/so3_core.c``,
  ``so3_sampling.c`` and ``so3_conv.c`` compiled unmodified against the same
  stand-ins (``make -C oracle ref``; needs the reference tree at build time).
  Optional: ``ref()`` returns None when it was not built.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "liboracle.so")
REFLIB = os.path.join(HERE, "_ref", "libso3ref.so")

MW, MWSS = 0, 1
ZERO_FIRST, NEGATIVE_FIRST = 0, 1
PADDED, COMPACT = 0, 1
ALL, EVEN, ODD, MAXIMUM, MODE_L = 0, 1, 2, 3, 4
RISBO, TRAPANI = 0, 1


class Params(ctypes.Structure):
    """so3_parameters_t (reference include/so3/so3_types.h:130-201)."""

    _fields_ = [
        ("verbosity", ctypes.c_int),
        ("reality", ctypes.c_int),
        ("L0", ctypes.c_int),
        ("L", ctypes.c_int),
        ("N", ctypes.c_int),
        ("sampling_scheme", ctypes.c_int),
        ("n_order", ctypes.c_int),
        ("storage", ctypes.c_int),
        ("n_mode", ctypes.c_int),
        ("dl_method", ctypes.c_int),
        ("steerable", ctypes.c_int),
    ]


def params(L, N, L0=0, reality=0, sampling=MW, order=NEGATIVE_FIRST, storage=PADDED,
           mode=ALL, method=RISBO, steerable=0) -> Params:
    return Params(0, reality, L0, L, N, sampling, order, storage, mode, method, steerable)


def f_size(p: Params) -> int:
    na = 2 * p.L - 1 if p.sampling_scheme == MW else 2 * p.L
    nb = p.L if p.sampling_scheme == MW else p.L + 1
    ng = p.N if p.steerable else 2 * p.N - 1
    return na * nb * ng


_P = ctypes.POINTER(Params)
_VP = ctypes.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def build(ref: bool = False) -> None:
    targets = ["lib"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB, mode=ctypes.RTLD_LOCAL)
        for name in ("oracle_inverse_via_ssht", "oracle_forward_via_ssht",
                     "oracle_inverse_via_ssht_real", "oracle_forward_via_ssht_real"):
            getattr(L, name).argtypes = [_VP, _VP, _P]
            getattr(L, name).restype = None
        L.oracle_harmonic_convolution.argtypes = [_VP, _P, _VP, _P, _VP, _P]
        L.oracle_s2toso3_harmonic_convolution.argtypes = [_VP, _P, _VP, _VP]
        L.oracle_convolved_parameters.argtypes = [_P, _P]
        L.oracle_convolved_parameters.restype = Params
        L.oracle_flmn_size.argtypes = [_P]
        L.oracle_elmn2ind.argtypes = [ctypes.c_int] * 3 + [_P]
        L.oracle_elmn2ind_real.argtypes = [ctypes.c_int] * 3 + [_P]
        L.oracle_dl_plane.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_dft_strided.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_long,
                                         ctypes.c_long, ctypes.c_int]
        _lib = L
    return _lib


def ref():
    """The reference C compiled against the stand-ins, or None if not built."""
    global _ref
    if _ref is None and os.path.exists(REFLIB):
        R = ctypes.CDLL(REFLIB, mode=ctypes.RTLD_LOCAL)
        for name in ("so3_core_inverse_via_ssht", "so3_core_forward_via_ssht",
                     "so3_core_inverse_via_ssht_real", "so3_core_forward_via_ssht_real",
                     "so3_core_inverse_direct", "so3_core_forward_direct",
                     "so3_core_inverse_direct_real", "so3_core_forward_direct_real",
                     "so3_adjoint_inverse_direct", "so3_adjoint_forward_direct",
                     "so3_adjoint_inverse_direct_real", "so3_adjoint_forward_direct_real"):
            getattr(R, name).argtypes = [_VP, _VP, _P]
            getattr(R, name).restype = None
        R.so3_conv_harmonic_convolution.argtypes = [_VP, _P, _VP, _P, _VP, _P]
        R.so3_conv_convolution.argtypes = [_VP, _P, _VP, _P, _VP, _P]
        R.so3_conv_s2toso3_harmonic_convolution.argtypes = [_VP, _P, _VP, _VP]
        R.so3_conv_get_parameters_of_convolved_lmn.argtypes = [_P, _P]
        R.so3_conv_get_parameters_of_convolved_lmn.restype = Params
        R.so3_sampling_flmn_size.argtypes = [_P]
        R.so3_sampling_f_size.argtypes = [_P]
        for nm in ("so3_sampling_elmn2ind", "so3_sampling_elmn2ind_real"):
            getattr(R, nm).argtypes = [ctypes.POINTER(ctypes.c_int)] + [ctypes.c_int] * 3 + [_P]
        for nm in ("so3_sampling_ind2elmn", "so3_sampling_ind2elmn_real"):
            getattr(R, nm).argtypes = [ctypes.POINTER(ctypes.c_int)] * 3 + [ctypes.c_int, _P]
        _ref = R
    return _ref


def flmn_size(p: Params) -> int:
    return lib().oracle_flmn_size(ctypes.byref(p))


def inverse(flmn: np.ndarray, p: Params) -> np.ndarray:
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    if p.reality:
        f = np.zeros(f_size(p), np.float64)
        lib().oracle_inverse_via_ssht_real(_ptr(f), _ptr(flmn), ctypes.byref(p))
    else:
        f = np.zeros(f_size(p), np.complex128)
        lib().oracle_inverse_via_ssht(_ptr(f), _ptr(flmn), ctypes.byref(p))
    return f


def forward(f: np.ndarray, p: Params, out: np.ndarray | None = None) -> np.ndarray:
    flmn = np.zeros(flmn_size(p), np.complex128) if out is None else out
    if p.reality:
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib().oracle_forward_via_ssht_real(_ptr(flmn), _ptr(f), ctypes.byref(p))
    else:
        f = np.ascontiguousarray(f, dtype=np.complex128)
        lib().oracle_forward_via_ssht(_ptr(flmn), _ptr(f), ctypes.byref(p))
    return flmn


def ref_inverse(flmn, p, direct=False):
    R = ref()
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    kind = "direct" if direct else "via_ssht"
    if p.reality:
        f = np.zeros(f_size(p), np.float64)
        getattr(R, f"so3_core_inverse_{kind}_real")(_ptr(f), _ptr(flmn), ctypes.byref(p))
    else:
        f = np.zeros(f_size(p), np.complex128)
        getattr(R, f"so3_core_inverse_{kind}")(_ptr(f), _ptr(flmn), ctypes.byref(p))
    return f


def ref_forward(f, p, direct=False):
    R = ref()
    flmn = np.zeros(R.so3_sampling_flmn_size(ctypes.byref(p)), np.complex128)
    kind = "direct" if direct else "via_ssht"
    if p.reality:
        f = np.ascontiguousarray(f, dtype=np.float64)
        getattr(R, f"so3_core_forward_{kind}_real")(_ptr(flmn), _ptr(f), ctypes.byref(p))
    else:
        f = np.ascontiguousarray(f, dtype=np.complex128)
        getattr(R, f"so3_core_forward_{kind}")(_ptr(flmn), _ptr(f), ctypes.byref(p))
    return flmn


def ref_adjoint_inverse(f, p):
    """The reference's so3_adjoint_inverse_direct (src/c/so3_adjoint.c:34)."""
    R = ref()
    flmn = np.zeros(R.so3_sampling_flmn_size(ctypes.byref(p)), np.complex128)
    f = np.ascontiguousarray(f, dtype=np.complex128)
    R.so3_adjoint_inverse_direct(_ptr(flmn), _ptr(f), ctypes.byref(p))
    return flmn


def ref_adjoint_forward(flmn, p):
    """The reference's so3_adjoint_forward_direct (src/c/so3_adjoint.c:402)."""
    R = ref()
    f = np.zeros(f_size(p), np.complex128)
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    R.so3_adjoint_forward_direct(_ptr(f), _ptr(flmn), ctypes.byref(p))
    return f


def ref_adjoint_inverse_real(f, p):
    """The reference's so3_adjoint_inverse_direct_real (src/c/so3_adjoint.c:939)."""
    R = ref()
    flmn = np.zeros(R.so3_sampling_flmn_size(ctypes.byref(p)), np.complex128)
    f = np.ascontiguousarray(f, dtype=np.float64)
    R.so3_adjoint_inverse_direct_real(_ptr(flmn), _ptr(f), ctypes.byref(p))
    return flmn


def ref_adjoint_forward_real(flmn, p):
    """The reference's so3_adjoint_forward_direct_real (src/c/so3_adjoint.c:1313)."""
    R = ref()
    f = np.zeros(f_size(p), np.float64)
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    R.so3_adjoint_forward_direct_real(_ptr(f), _ptr(flmn), ctypes.byref(p))
    return f


def harmonic_convolution(flmn, fp: Params, glmn, gp: Params):
    hp = lib().oracle_convolved_parameters(ctypes.byref(fp), ctypes.byref(gp))
    h = np.zeros(flmn_size(hp), np.complex128)
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    glmn = np.ascontiguousarray(glmn, dtype=np.complex128)
    lib().oracle_harmonic_convolution(_ptr(h), ctypes.byref(hp), _ptr(flmn), ctypes.byref(fp),
                                      _ptr(glmn), ctypes.byref(gp))
    return h, hp


def s2toso3(hp: Params, flm, glm):
    h = np.zeros(flmn_size(hp), np.complex128)
    flm = np.ascontiguousarray(flm, dtype=np.complex128)
    glm = np.ascontiguousarray(glm, dtype=np.complex128)
    lib().oracle_s2toso3_harmonic_convolution(_ptr(h), ctypes.byref(hp), _ptr(flm), _ptr(glm))
    return h


def dl_plane(L: int, el: int, method: int) -> np.ndarray:
    out = np.zeros((el + 1, el + 1), np.float64)
    lib().oracle_dl_plane(_ptr(out), L, el, method)
    return out


def dft_strided(x: np.ndarray, n: int, howmany: int, stride: int, dist: int, sign: int):
    x = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().oracle_dft_strided(_ptr(x), n, howmany, stride, dist, sign)
    return x
