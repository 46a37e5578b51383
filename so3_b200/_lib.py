"""ctypes binding of libso3gpu.so (the C ABI declared in include/so3/*.h and
include/so3gpu.h).  The library is loaded from the package's lib/ directory;
a missing library raises immediately -- there is no CPU fallback."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libso3gpu.so")


class Params(ctypes.Structure):
    """so3_parameters_t (include/so3/so3_types.h)."""

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


class SO3Error(RuntimeError):
    pass


_P = ctypes.POINTER(Params)
_VP = ctypes.c_void_p
_IP = ctypes.POINTER(ctypes.c_int)
_I = ctypes.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "so3_core_inverse_via_ssht": (None, [_VP, _VP, _P]),
    "so3_core_inverse_via_ssht_real": (None, [_VP, _VP, _P]),
    "so3_core_forward_via_ssht": (None, [_VP, _VP, _P]),
    "so3_core_forward_via_ssht_real": (None, [_VP, _VP, _P]),
    "so3_core_inverse_direct": (None, [_VP, _VP, _P]),
    "so3_core_inverse_direct_real": (None, [_VP, _VP, _P]),
    "so3_core_forward_direct": (None, [_VP, _VP, _P]),
    "so3_core_forward_direct_real": (None, [_VP, _VP, _P]),
    "so3_adjoint_inverse_direct": (None, [_VP, _VP, _P]),
    "so3_adjoint_forward_direct": (None, [_VP, _VP, _P]),
    "so3_conv_convolution": (None, [_VP, _P, _VP, _P, _VP, _P]),
    "so3_conv_harmonic_convolution": (None, [_VP, _P, _VP, _P, _VP, _P]),
    "so3_conv_get_parameters_of_convolved_lmn": (Params, [_P, _P]),
    "so3_conv_get_parameters_of_convolved_lmn_void": (None, [_P, _P, _P]),
    "so3_conv_s2toso3_harmonic_convolution": (None, [_VP, _P, _VP, _VP]),
    "so3_sampling_weight": (None, None),  # complex return: not called through ctypes
    "so3_sampling_f_size": (_I, [_P]),
    "so3_sampling_n": (_I, [_P]),
    "so3_sampling_nalpha": (_I, [_P]),
    "so3_sampling_nbeta": (_I, [_P]),
    "so3_sampling_ngamma": (_I, [_P]),
    "so3_sampling_a2alpha": (ctypes.c_double, [_I, _P]),
    "so3_sampling_b2beta": (ctypes.c_double, [_I, _P]),
    "so3_sampling_g2gamma": (ctypes.c_double, [_I, _P]),
    "so3_sampling_flmn_size": (_I, [_P]),
    "so3_sampling_elmn2ind": (None, [_IP, _I, _I, _I, _P]),
    "so3_sampling_ind2elmn": (None, [_IP, _IP, _IP, _I, _P]),
    "so3_sampling_elmn2ind_real": (None, [_IP, _I, _I, _I, _P]),
    "so3_sampling_ind2elmn_real": (None, [_IP, _IP, _IP, _I, _P]),
    "so3_sampling_n_loop_values": (None, [_IP, _IP, _IP, _P]),
    "so3_sampling_el_loop_values": (None, [_IP, _IP, _IP, _I, _P]),
    "so3_sampling_m_loop_values": (None, [_IP, _IP, _IP, _I]),
    "so3_sampling_is_elmn_non_zero": (ctypes.c_bool, [_I, _I, _I, _P]),
    "so3_sampling_is_elmn_non_zero_return_int": (_I, [_I, _I, _I, _P]),
    "so3gpu_context_create": (_VP, [_I, _VP]),
    "so3gpu_context_destroy": (None, [_VP]),
    "so3gpu_context_set_stream": (_I, [_VP, _VP]),
    "so3gpu_prepare": (_I, [_VP, _P]),
    "so3gpu_workspace_size": (ctypes.c_size_t, [_P]),
    "so3gpu_inverse": (_I, [_VP, _VP, _VP, _P]),
    "so3gpu_forward": (_I, [_VP, _VP, _VP, _P]),
    "so3gpu_inverse_real": (_I, [_VP, _VP, _VP, _P]),
    "so3gpu_forward_real": (_I, [_VP, _VP, _VP, _P]),
    "so3gpu_s2toso3_harmonic_convolution": (_I, [_VP, _VP, _P, _VP, _VP]),
    "so3gpu_harmonic_convolution": (_I, [_VP, _VP, _P, _VP, _P, _VP, _P]),
    "so3gpu_stage_timing": (_I, [_VP, _I]),
    "so3gpu_stage_times": (_I, [_VP, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong), _I]),
    "so3gpu_get_stage_variants": (_I, [_I, _P, _VP]),
    "so3gpu_inverse_batch": (_I, [_VP, _VP, _VP, _I, _P, _I]),
    "so3gpu_inverse_ragged": (_I, [_VP, _VP, _VP, _VP, _I, _I]),
    "so3gpu_forward_ragged": (_I, [_VP, _VP, _VP, _VP, _I, _I]),
    "so3gpu_s2toso3_inverse_batch": (_I, [_VP, _VP, _VP, _VP, _I, _P, _I]),
    "so3gpu_server_create": (_VP, [_I, ctypes.c_size_t, _I, _I, _I]),
    "so3gpu_server_destroy": (None, [_VP]),
    "so3gpu_server_submit": (ctypes.c_longlong, [_VP, _I, _P, _VP, _VP, _VP, _I]),
    "so3gpu_server_poll": (_I, [_VP, ctypes.c_longlong, _VP, _VP, _VP, _VP]),
    "so3gpu_server_wait": (_I, [_VP, ctypes.c_longlong, _VP, _VP, _VP, _VP]),
    "so3gpu_server_drain": (None, [_VP]),
    "so3gpu_server_stats": (None, [_VP, _VP, _VP, _VP, _VP]),
    "so3gpu_forward_batch": (_I, [_VP, _VP, _VP, _I, _P, _I]),
    "so3gpu_set_stage_variants": (_I, [_I, _P, _VP]),
    "so3gpu_inverse_noalloc": (_I, [_VP, _VP, _P, _VP]),
    "so3gpu_last_status": (_I, []),
    "so3gpu_last_error": (ctypes.c_char_p, []),
    "so3gpu_set_error_mode": (None, [_I]),
    "so3gpu_launch_count": (ctypes.c_longlong, []),
    "so3gpu_take_kernel_error": (ctypes.c_int, []),
}

_lib = None


def load() -> ctypes.CDLL:
    """Loads libso3gpu.so (switching its errors to return-and-record)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SO3Error(f"libso3gpu.so not built ({LIB_PATH}); run python -m so3_b200.build")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        if args is not None:
            fn.restype = res
            fn.argtypes = args
    lib.so3gpu_set_error_mode(1)
    _lib = lib
    return lib


def check(what: str = "") -> None:
    lib = load()
    st = lib.so3gpu_last_status()
    if st != 0:
        msg = lib.so3gpu_last_error().decode(errors="replace")
        raise SO3Error(f"{what}: status {st}: {msg}")
