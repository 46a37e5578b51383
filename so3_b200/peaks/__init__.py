"""Throughput probes of the benchmark (FP64 FMA chain, int8 tcgen05.mma,
HBM copy), built from peaks.cu into so3_b200/lib/libso3peaks.so.  Loaded by
bench.py only; not part of the product library."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libso3peaks.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} missing: run python -m so3_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        for name in ("so3peaks_fp64_tflops", "so3peaks_int8_mma_tops", "so3peaks_hbm_copy_gbs",
                     "so3peaks_dmma_tflops"):
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _checked(v, what):
    if v < 0:
        raise RuntimeError(f"{what}: CUDA error in the probe")
    return v


def fp64_tflops(device: int = 0) -> float:
    """Measured FP64 FMA throughput of the device (TFLOP/s)."""
    return _checked(_load().so3peaks_fp64_tflops(device), "fp64 probe")


def int8_mma_tops(device: int = 0) -> float:
    """Measured tcgen05.mma kind::i8 (M=128, N=256) throughput (TOP/s)."""
    return _checked(_load().so3peaks_int8_mma_tops(device), "int8 tensor-core probe")


def hbm_copy_gbs(device: int = 0) -> float:
    """Measured device-to-device copy bandwidth (GB/s, read + write)."""
    return _checked(_load().so3peaks_hbm_copy_gbs(device), "HBM copy probe")


def dmma_tflops(device: int = 0) -> float:
    """Measured FP64 tensor-core (mma.sync m8n8k4 f64) throughput (TFLOP/s)."""
    return _checked(_load().so3peaks_dmma_tflops(device), "FP64 tensor-core probe")
