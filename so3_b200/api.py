"""Python host API over libso3gpu, mirroring the reference's Cython binding
(src/so3/bindings.pyx:95-445): the same parameter class and helper names, the
same argument meaning, numpy in / numpy out.  Every transform runs on the GPU
through the C ABI; ``*_device`` variants take torch CUDA tensors and skip the
host copies.
"""
from __future__ import annotations

import ctypes
from typing import Iterator

import numpy as np

from . import _lib
from ._lib import Params, SO3Error

SO3_SAMPLING_MW, SO3_SAMPLING_MW_SS = 0, 1
SO3_N_ORDER_ZERO_FIRST, SO3_N_ORDER_NEGATIVE_FIRST = 0, 1
SO3_STORAGE_PADDED, SO3_STORAGE_COMPACT = 0, 1
(SO3_N_MODE_ALL, SO3_N_MODE_EVEN, SO3_N_MODE_ODD, SO3_N_MODE_MAXIMUM, SO3_N_MODE_L) = range(5)
SSHT_DL_RISBO, SSHT_DL_TRAPANI = 0, 1


class SO3Parameters:
    """Parameter object with the reference binding's defaults (bindings.pyx:95-137)."""

    def __init__(self, L=32, N=4, L0=0, verbosity=0, reality=0, sampling_scheme=SO3_SAMPLING_MW,
                 n_order=SO3_N_ORDER_NEGATIVE_FIRST, storage=SO3_STORAGE_PADDED, n_mode=SO3_N_MODE_ALL,
                 dl_method=SSHT_DL_RISBO, steerable=0):
        self.L, self.N, self.L0 = L, N, L0
        self.verbosity, self.reality = verbosity, reality
        self.sampling_scheme, self.n_order, self.storage = sampling_scheme, n_order, storage
        self.n_mode, self.dl_method, self.steerable = n_mode, dl_method, steerable

    def from_dict(self, d: dict) -> "SO3Parameters":
        for k in ("L", "N", "L0", "verbosity", "reality", "sampling_scheme", "n_order", "storage",
                  "n_mode", "dl_method", "steerable"):
            setattr(self, k, d[k])
        return self

    def to_struct(self) -> Params:
        return Params(self.verbosity, self.reality, self.L0, self.L, self.N, self.sampling_scheme,
                      self.n_order, self.storage, self.n_mode, self.dl_method, self.steerable)

    @staticmethod
    def from_struct(p: Params) -> "SO3Parameters":
        return SO3Parameters(p.L, p.N, p.L0, p.verbosity, p.reality, p.sampling_scheme, p.n_order, p.storage,
                             p.n_mode, p.dl_method, p.steerable)

    def __repr__(self):
        return (f"SO3Parameters(L={self.L}, N={self.N}, L0={self.L0}, reality={self.reality}, "
                f"sampling={self.sampling_scheme}, order={self.n_order}, storage={self.storage}, "
                f"n_mode={self.n_mode}, dl_method={self.dl_method}, steerable={self.steerable})")


def create_parameter_dict(L, N, L0=0, verbosity=0, reality=0, sampling_scheme_str="SO3_SAMPLING_MW",
                          n_order_str="SO3_N_ORDER_NEGATIVE_FIRST", storage_str="SO3_STORAGE_PADDED",
                          n_mode_str="SO3_N_MODE_ALL", dl_method_str="SSHT_DL_RISBO", steerable=0):
    """Same string-keyed constructor as bindings.pyx:140-214."""
    modes = {"SO3_N_MODE_ALL": 0, "SO3_N_MODE_EVEN": 1, "SO3_N_MODE_ODD": 2, "SO3_N_MODE_MAXIMUM": 3}
    return SO3Parameters(
        L=L, N=N, L0=L0, verbosity=verbosity, reality=reality,
        sampling_scheme=SO3_SAMPLING_MW if sampling_scheme_str == "SO3_SAMPLING_MW" else SO3_SAMPLING_MW_SS,
        n_order=SO3_N_ORDER_NEGATIVE_FIRST if n_order_str == "SO3_N_ORDER_NEGATIVE_FIRST" else SO3_N_ORDER_ZERO_FIRST,
        storage=SO3_STORAGE_PADDED if storage_str == "SO3_STORAGE_PADDED" else SO3_STORAGE_COMPACT,
        n_mode=modes.get(n_mode_str, SO3_N_MODE_L),
        dl_method=SSHT_DL_RISBO if dl_method_str == "SSHT_DL_RISBO" else SSHT_DL_TRAPANI,
        steerable=steerable)


def _s(p) -> Params:
    return p.to_struct() if isinstance(p, SO3Parameters) else p


def _checked(p) -> Params:
    """Struct for a transform call.  The C sampling helpers exit the process on
    an invalid sampling scheme, storage or n-order (reference behaviour), so
    the Python layer rejects those first."""
    q = _s(p)
    if q.sampling_scheme not in (0, 1):
        raise SO3Error("status 1: Invalid sampling scheme.")
    if q.storage not in (0, 1):
        raise SO3Error("status 1: Invalid storage method.")
    if q.n_order not in (0, 1):
        raise SO3Error("status 1: Invalid n-order.")
    return q


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ------------------------------------------------------------ sampling helpers
def f_size(p) -> int:
    return _lib.load().so3_sampling_f_size(ctypes.byref(_s(p)))


def n_alpha(p) -> int:
    return _lib.load().so3_sampling_nalpha(ctypes.byref(_s(p)))


def n_beta(p) -> int:
    return _lib.load().so3_sampling_nbeta(ctypes.byref(_s(p)))


def n_gamma(p) -> int:
    return _lib.load().so3_sampling_ngamma(ctypes.byref(_s(p)))


def flmn_size(p) -> int:
    return _lib.load().so3_sampling_flmn_size(ctypes.byref(_s(p)))


def elmn2ind(el, m, n, p) -> int:
    q = _s(p)
    ind = ctypes.c_int()
    fn = _lib.load().so3_sampling_elmn2ind_real if q.reality == 1 else _lib.load().so3_sampling_elmn2ind
    fn(ctypes.byref(ind), el, m, n, ctypes.byref(q))
    return ind.value


def ind2elmn(ind, p):
    q = _s(p)
    el, m, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    fn = _lib.load().so3_sampling_ind2elmn_real if q.reality == 1 else _lib.load().so3_sampling_ind2elmn
    fn(ctypes.byref(el), ctypes.byref(m), ctypes.byref(n), ind, ctypes.byref(q))
    return el.value, m.value, n.value


def get_loop_n_values(p):
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _lib.load().so3_sampling_n_loop_values(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(_s(p)))
    return a.value, b.value, c.value


def loop_over_n(p) -> Iterator[int]:
    s, e, i = get_loop_n_values(p)
    yield from range(s, e + 1, i)


def get_loop_el_values(n, p):
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _lib.load().so3_sampling_el_loop_values(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), n,
                                            ctypes.byref(_s(p)))
    return a.value, b.value, c.value


def loop_over_el(n, p) -> Iterator[int]:
    s, e, i = get_loop_el_values(n, p)
    yield from range(s, e + 1, i)


def get_loop_m_values(el):
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _lib.load().so3_sampling_m_loop_values(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), el)
    return a.value, b.value, c.value


def loop_over_m(el) -> Iterator[int]:
    s, e, i = get_loop_m_values(el)
    yield from range(s, e + 1, i)


def is_elmn_non_zero(el, m, n, p) -> bool:
    return bool(_lib.load().so3_sampling_is_elmn_non_zero_return_int(el, m, n, ctypes.byref(_s(p))))


# ------------------------------------------------------------ transforms (host)
def inverse(flmn: np.ndarray, p) -> np.ndarray:
    """bindings.pyx:315-336: flmn -> samples (complex, or real when p.reality)."""
    q = _checked(p)
    lib = _lib.load()
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    if q.reality:
        f = np.zeros(f_size(q), np.float64)
        lib.so3_core_inverse_via_ssht_real(_ptr(f), _ptr(flmn), ctypes.byref(q))
    else:
        f = np.zeros(f_size(q), np.complex128)
        lib.so3_core_inverse_via_ssht(_ptr(f), _ptr(flmn), ctypes.byref(q))
    _lib.check("inverse")
    return f


def forward(f: np.ndarray, p) -> np.ndarray:
    """bindings.pyx:338-357: samples -> flmn; a real array needs p.reality."""
    q = _checked(p)
    lib = _lib.load()
    flmn = np.zeros(flmn_size(q), np.complex128)
    if np.isrealobj(f):
        if not q.reality:
            raise ValueError("f has a real data type but reality flag not set")
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib.so3_core_forward_via_ssht_real(_ptr(flmn), _ptr(f), ctypes.byref(q))
    else:
        f = np.ascontiguousarray(f, dtype=np.complex128)
        lib.so3_core_forward_via_ssht(_ptr(flmn), _ptr(f), ctypes.byref(q))
    _lib.check("forward")
    return flmn


def adjoint_inverse(f: np.ndarray, p) -> np.ndarray:
    """Adjoint of the inverse transform: samples -> coefficients, MW
    (so3_adjoint_inverse_direct, reference src/c/so3_adjoint.c:34; with
    p.reality, so3_adjoint_inverse_direct_real, :939, on real samples)."""
    q = _checked(p)
    flmn = np.zeros(flmn_size(q), np.complex128)
    lib = _lib.load()
    if q.reality:
        f = np.ascontiguousarray(f, dtype=np.float64)
        lib.so3_adjoint_inverse_direct_real(_ptr(flmn), _ptr(f), ctypes.byref(q))
    else:
        f = np.ascontiguousarray(f, dtype=np.complex128)
        lib.so3_adjoint_inverse_direct(_ptr(flmn), _ptr(f), ctypes.byref(q))
    _lib.check("adjoint_inverse")
    return flmn


def adjoint_forward(flmn: np.ndarray, p) -> np.ndarray:
    """Adjoint of the forward transform: coefficients -> samples, MW
    (so3_adjoint_forward_direct, reference src/c/so3_adjoint.c:402; with
    p.reality, so3_adjoint_forward_direct_real, :1313, to real samples)."""
    q = _checked(p)
    lib = _lib.load()
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    if q.reality:
        f = np.zeros(f_size(q), np.float64)
        lib.so3_adjoint_forward_direct_real(_ptr(f), _ptr(flmn), ctypes.byref(q))
    else:
        f = np.zeros(f_size(q), np.complex128)
        lib.so3_adjoint_forward_direct(_ptr(f), _ptr(flmn), ctypes.byref(q))
    _lib.check("adjoint_forward")
    return f


def get_convolved_parameters(fp, gp) -> SO3Parameters:
    h = Params()
    _lib.load().so3_conv_get_parameters_of_convolved_lmn_void(ctypes.byref(h), ctypes.byref(_s(fp)),
                                                              ctypes.byref(_s(gp)))
    _lib.check("get_convolved_parameters")
    return SO3Parameters.from_struct(h)


def convolve(f, fp, g, gp):
    """bindings.pyx:380-409: real-space convolution of two sampled signals."""
    hp = get_convolved_parameters(fp, gp)
    h = np.zeros(f_size(hp), np.complex128)
    f = np.ascontiguousarray(f, dtype=np.complex128)
    g = np.ascontiguousarray(g, dtype=np.complex128)
    _lib.load().so3_conv_convolution(_ptr(h), ctypes.byref(hp.to_struct()), _ptr(f), ctypes.byref(_s(fp)),
                                     _ptr(g), ctypes.byref(_s(gp)))
    _lib.check("convolve")
    return h, hp


def convolve_harmonic(flmn, fp, glmn, gp):
    """Harmonic-space SO(3) convolution h_lmn = sum_k f_lmk conj(g_lnk).

    The reference binding (bindings.pyx:411-432) routes this name to the
    real-space so3_conv_convolution by mistake; this implementation calls the
    harmonic convolution (src/c/so3_conv.c:44-90) the name describes.
    """
    hp = get_convolved_parameters(fp, gp)
    h = np.zeros(flmn_size(hp), np.complex128)
    flmn = np.ascontiguousarray(flmn, dtype=np.complex128)
    glmn = np.ascontiguousarray(glmn, dtype=np.complex128)
    _lib.load().so3_conv_harmonic_convolution(_ptr(h), ctypes.byref(hp.to_struct()), _ptr(flmn),
                                              ctypes.byref(_s(fp)), _ptr(glmn), ctypes.byref(_s(gp)))
    _lib.check("convolve_harmonic")
    return h, hp


def s2toso3_harmonic_convolution(hp, flm, glm):
    """bindings.pyx:434-445."""
    q = _s(hp)
    h = np.zeros(flmn_size(q), np.complex128)
    flm = np.ascontiguousarray(flm, dtype=np.complex128)
    glm = np.ascontiguousarray(glm, dtype=np.complex128)
    _lib.load().so3_conv_s2toso3_harmonic_convolution(_ptr(h), ctypes.byref(q), _ptr(flm), _ptr(glm))
    _lib.check("s2toso3_harmonic_convolution")
    return h


# ------------------------------------------------------------ device (torch) API
class Context:
    """so3gpu_context bound to one device and a torch CUDA stream."""

    def __init__(self, device: int = 0, stream=None):
        self._lib = _lib.load()
        handle = stream.cuda_stream if stream is not None else None
        self._c = self._lib.so3gpu_context_create(device, handle)
        if not self._c:
            _lib.check("context_create")
        self.device = device

    def close(self):
        if getattr(self, "_c", None):
            self._lib.so3gpu_context_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        self._lib.so3gpu_context_set_stream(self._c, stream.cuda_stream if stream is not None else None)

    def prepare(self, p):
        q = _s(p)
        if self._lib.so3gpu_prepare(self._c, ctypes.byref(q)):
            _lib.check("prepare")

    def inverse(self, flmn, p, out=None):
        import torch
        q = _s(p)
        if out is None:
            out = torch.empty(f_size(q), dtype=torch.float64 if q.reality else torch.complex128, device=flmn.device)
        fn = self._lib.so3gpu_inverse_real if q.reality else self._lib.so3gpu_inverse
        if fn(self._c, out.data_ptr(), flmn.data_ptr(), ctypes.byref(q)):
            _lib.check("so3gpu_inverse")
        return out

    def forward(self, f, p, out=None):
        import torch
        q = _s(p)
        if out is None:
            out = torch.zeros(flmn_size(q), dtype=torch.complex128, device=f.device)
        fn = self._lib.so3gpu_forward_real if q.reality else self._lib.so3gpu_forward
        if fn(self._c, out.data_ptr(), f.data_ptr(), ctypes.byref(q)):
            _lib.check("so3gpu_forward")
        return out

    def _batch(self, fn, ins, outs, q, precision, name):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        n = len(ins)
        pin = (ctypes.c_void_p * n)(*[t.data_ptr() for t in ins])
        pout = (ctypes.c_void_p * n)(*[t.data_ptr() for t in outs])
        if fn(self._c, pout, pin, n, ctypes.byref(q), PRECISIONS[precision]):
            _lib.check(name)
        return outs

    def inverse_batch(self, flmns, p, precision="fp64", outs=None):
        """Inverse transforms of a list of coefficient tensors with one
        parameter set; precision "fp64" or "mixed" (int8 split contractions)."""
        import torch
        q = _s(p)
        if outs is None:
            dt = torch.float64 if q.reality else torch.complex128
            outs = [torch.empty(f_size(q), dtype=dt, device=x.device) for x in flmns]
        return self._batch(self._lib.so3gpu_inverse_batch, flmns, outs, q, precision, "so3gpu_inverse_batch")

    def forward_batch(self, fs, p, precision="fp64", outs=None):
        import torch
        q = _s(p)
        if outs is None:
            outs = [torch.zeros(flmn_size(q), dtype=torch.complex128, device=x.device) for x in fs]
        return self._batch(self._lib.so3gpu_forward_batch, fs, outs, q, precision, "so3gpu_forward_batch")

    def _ragged(self, fn, ins, outs, ps, precision, name):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        n = len(ins)
        arr = (Params * n)(*[_s(p) for p in ps])
        pin = (ctypes.c_void_p * n)(*[t.data_ptr() for t in ins])
        pout = (ctypes.c_void_p * n)(*[t.data_ptr() for t in outs])
        if fn(self._c, pout, pin, arr, n, PRECISIONS[precision]):
            _lib.check(name)
        return outs

    def inverse_ragged(self, flmns, ps, precision="fp64", outs=None):
        """Inverse transforms of signals with one parameter set each (ps[k]);
        "mixed" runs every complex signal's contraction in one ragged
        tensor-core launch."""
        import torch
        if outs is None:
            outs = [torch.empty(f_size(p), dtype=torch.float64 if p.reality else torch.complex128, device=x.device)
                    for x, p in zip(flmns, ps)]
        return self._ragged(self._lib.so3gpu_inverse_ragged, flmns, outs, ps, precision, "so3gpu_inverse_ragged")

    def forward_ragged(self, fs, ps, precision="fp64", outs=None):
        import torch
        if outs is None:
            outs = [torch.zeros(flmn_size(p), dtype=torch.complex128, device=x.device) for x, p in zip(fs, ps)]
        return self._ragged(self._lib.so3gpu_forward_ragged, fs, outs, ps, precision, "so3gpu_forward_ragged")

    def s2toso3_inverse_batch(self, hp, flm, glms, precision="fp64", outs=None):
        """Samples of the directional convolutions of flm with each kernel in
        glms (so3_conv_s2toso3_harmonic_convolution with parameters hp, then
        the inverse transform); precision "fp64" or "mixed"."""
        import torch
        q = _s(hp)
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        if outs is None:
            outs = [torch.empty(f_size(q), dtype=torch.complex128, device=flm.device) for _ in glms]
        n = len(glms)
        pg = (ctypes.c_void_p * n)(*[t.data_ptr() for t in glms])
        pf = (ctypes.c_void_p * n)(*[t.data_ptr() for t in outs])
        if self._lib.so3gpu_s2toso3_inverse_batch(self._c, pf, ctypes.c_void_p(flm.data_ptr()), pg, n,
                                                  ctypes.byref(q), PRECISIONS[precision]):
            _lib.check("so3gpu_s2toso3_inverse_batch")
        return outs

    def s2toso3(self, hp, flm, glm, out=None):
        import torch
        q = _s(hp)
        if out is None:
            out = torch.empty(flmn_size(q), dtype=torch.complex128, device=flm.device)
        if self._lib.so3gpu_s2toso3_harmonic_convolution(self._c, out.data_ptr(), ctypes.byref(q), flm.data_ptr(),
                                                         glm.data_ptr()):
            _lib.check("so3gpu_s2toso3_harmonic_convolution")
        return out


    def stage_timing(self, enable: bool = True):
        self._lib.so3gpu_stage_timing(self._c, 1 if enable else 0)

    def stage_times(self):
        """{stage name: (total ms, launches)} since the previous call."""
        ms = (ctypes.c_double * 16)()
        cnt = (ctypes.c_longlong * 16)()
        if self._lib.so3gpu_stage_times(self._c, ms, cnt, 16):
            _lib.check("stage_times")
        return {name: (ms[i], cnt[i]) for i, name in enumerate(STAGES) if cnt[i]}


STAGES = ["inv_contract", "inv_beta", "inv_alpha", "inv_gamma", "fwd_gamma", "fwd_alpha", "fwd_beta_conv",
          "fwd_contract", "mixed_inv_contract", "mixed_fwd_contract", "mixed_fwd_beta"]

PRECISIONS = {"fp64": 0, "mixed": 1}


def workspace_size(p) -> int:
    return _lib.load().so3gpu_workspace_size(ctypes.byref(_s(p)))


def launch_count() -> int:
    return _lib.load().so3gpu_launch_count()


def take_kernel_error() -> int:
    """Reads and clears the tensor-core kernels' wait-timeout flag of the
    current device (0: none)."""
    return _lib.load().so3gpu_take_kernel_error()


__all__ = [n for n in dir() if not n.startswith("_")] + ["SO3Error"]
