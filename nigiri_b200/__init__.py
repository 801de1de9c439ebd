"""B200-native RAPTOR engine behind nigiri's routing seam.

The product is the C ABI of include/b2r.h implemented by libb2r.so
(hand-written sm_100a CUDA kernels + host driver).  This package holds the
build recipe, the ctypes mirror of the ABI and a Python rendering of
nigiri's routing interface (nigiri_b200.routing).
"""
from . import _abi  # noqa: F401

__all__ = ["_abi", "routing", "timetable"]
