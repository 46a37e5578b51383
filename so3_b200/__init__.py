"""B200-native implementation of the SO3 library's exact Wigner transform path.

The product is the C ABI in so3_b200/lib/libso3gpu.so (headers in include/):
drop-in so3_core_* / so3_conv_* / so3_sampling_* entry points plus the
so3gpu_* device API, backed by sm_100a kernels.  This package is the Python
host side: ``so3_b200.api`` mirrors the reference's Python binding.
"""
from .api import *  # noqa: F401,F403
from .api import SO3Error, SO3Parameters  # noqa: F401

__version__ = "0.1.0"
