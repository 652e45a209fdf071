"""nanomap_b200 -- B200-native NanoMap mapping and simulation path.

The product is the C ABI in include/nanomap_b200.h, implemented by libnanomap_b200.so (CUDA
kernels for sm_100a plus C++ host code).  This package holds its sources (csrc/), the build
step (build.py), the ctypes view used by the tests and the benchmark (api.py), and the seeded
scene generator (scenes.py).
"""
from . import _native  # noqa: F401

__all__ = ["_native"]
