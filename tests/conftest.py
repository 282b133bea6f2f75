"""Shared test setup: markers, library loading, oracle handles.

`-m "not gpu"` tests need no GPU; `-m gpu` tests run the CUDA kernels through
the C ABI and compare them with the oracle (oracle/liboracle.so) and, where
it is built, the reference's own CPU callbacks (oracle/_ref/).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100) device")


def _make(path: str) -> None:
    subprocess.run(["make", "-s", "-C", path], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def oracle():
    lib_path = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib_path):
        _make(os.path.join(ROOT, "oracle"))
    lib = ctypes.CDLL(lib_path)
    lib.orc_set_threads(min(8, os.cpu_count() or 1))
    return lib


@pytest.fixture(scope="session")
def ref_imgf():
    """The reference's own imageFilter CPU callbacks, if oracle/_ref was built."""
    path = os.path.join(ROOT, "oracle", "_ref", "libref_imgf.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    return ctypes.CDLL(path)


@pytest.fixture(scope="session")
def pmb():
    from unicorn_b200 import capi

    return capi.lib()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    return torch


def ptr(a: np.ndarray) -> ctypes.c_void_p:
    return a.ctypes.data_as(ctypes.c_void_p)
