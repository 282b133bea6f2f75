"""unicorn_b200: B200-native (sm_100a) rebuild of Unicorn/pmlib's single-device
CUDA subtask execution path and the testSuite apps' subtask kernels.

The product is native: libpmb.so (C ABI, CUDA kernels) and libpmlib.so (the
pm:: C++ API runtime).  This Python package only binds the C ABI for tests and
benchmarks (`unicorn_b200.capi`) and offers thin array-level wrappers
(`unicorn_b200.ops`).
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
