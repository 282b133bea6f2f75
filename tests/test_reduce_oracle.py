"""CPU checks of the oracle's restatement of the reference reducer
(pmReducer::ReduceMemories, source/code/src/pmReducer.cpp:590-700) on
hand-computed cases, and the shared input generator of the GPU parity test.
The cases spell out the operations' edge semantics (LOGICAL_XOR is a != b;
bitwise operations on floats act on the values converted to unsigned
integers; MIN/MAX are std::min/std::max); tests/test_reduce_ref.py checks the
restatement bit for bit against the reference's own ReduceMemories."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ptr

DTYPES = {"int32": (0, np.dtype(np.int32)), "uint32": (1, np.dtype(np.uint32)), "int64": (2, np.dtype(np.int64)),
          "uint64": (3, np.dtype(np.uint64)), "float32": (4, np.dtype(np.float32)),
          "float64": (5, np.dtype(np.float64))}


def values(dt, op, n, seed):
    """Seeded inputs suited to the operation (small for PRODUCT, 0/1/2 for
    the logical operations, non-negative integral values for bitwise ones on
    floats)."""
    rng = np.random.default_rng(seed * 1000 + op)
    if op in (4, 6, 8):
        return rng.integers(0, 3, n).astype(dt)
    if op == 3:
        return rng.integers(1, 3, n).astype(dt)
    if dt.kind == "f":
        if op in (5, 7, 9):
            return rng.integers(0, 1 << 20, n).astype(dt)
        return ((rng.random(n) - 0.5) * 2000).astype(dt)
    info = np.iinfo(dt)
    return rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)


def oracle_fold(oracle, op, type_code, srcs):
    acc = srcs[0].copy()
    for s in srcs[1:]:
        assert oracle.orc_reduce_fold(op, type_code, ptr(acc), ptr(s), ctypes.c_size_t(acc.size)) == 0
    return acc


@pytest.mark.parametrize("type_name", list(DTYPES))
def test_add_min_max_product(oracle, type_name):
    type_code, dt = DTYPES[type_name]
    a = np.array([3, 7, 2, 9], dt)
    b = np.array([5, 1, 2, 4], dt)
    assert np.array_equal(oracle_fold(oracle, 0, type_code, [a, b]), np.array([8, 8, 4, 13], dt))
    assert np.array_equal(oracle_fold(oracle, 1, type_code, [a, b]), np.array([3, 1, 2, 4], dt))
    assert np.array_equal(oracle_fold(oracle, 2, type_code, [a, b]), np.array([5, 7, 2, 9], dt))
    assert np.array_equal(oracle_fold(oracle, 3, type_code, [a, b]), np.array([15, 7, 4, 36], dt))


@pytest.mark.parametrize("type_name", list(DTYPES))
def test_logical_and_bitwise(oracle, type_name):
    type_code, dt = DTYPES[type_name]
    a = np.array([0, 2, 3, 6], dt)
    b = np.array([0, 0, 5, 3], dt)
    assert np.array_equal(oracle_fold(oracle, 4, type_code, [a, b]), np.array([0, 0, 1, 1], dt))  # LOGICAL_AND
    assert np.array_equal(oracle_fold(oracle, 6, type_code, [a, b]), np.array([0, 1, 1, 1], dt))  # LOGICAL_OR
    assert np.array_equal(oracle_fold(oracle, 8, type_code, [a, b]), np.array([0, 1, 1, 1], dt))  # a != b
    assert np.array_equal(oracle_fold(oracle, 8, type_code, [a, a]), np.zeros(4, dt))
    assert np.array_equal(oracle_fold(oracle, 5, type_code, [a, b]), np.array([0, 0, 1, 2], dt))  # 3&5, 6&3
    assert np.array_equal(oracle_fold(oracle, 7, type_code, [a, b]), np.array([0, 2, 7, 7], dt))
    assert np.array_equal(oracle_fold(oracle, 9, type_code, [a, b]), np.array([0, 2, 6, 5], dt))


def test_bitwise_on_floats_converts_values(oracle):
    """2.75 | 4.5 acts on 2 and 4 (value conversion), not on the bit patterns."""
    a = np.array([2.75], np.float32)
    b = np.array([4.5], np.float32)
    assert oracle_fold(oracle, 7, 4, [a, b])[0] == 6.0


def test_float_sum_is_sequential(oracle):
    """Folding in order: (1e8 + 1) + (-1e8) in float32 is 0, not 1."""
    srcs = [np.array([1e8], np.float32), np.array([1.0], np.float32), np.array([-1e8], np.float32)]
    assert oracle_fold(oracle, 0, 4, srcs)[0] == 0.0


def test_rejects_unknown_codes(oracle):
    a = np.zeros(1, np.int32)
    assert oracle.orc_reduce_fold(10, 0, ptr(a), ptr(a), ctypes.c_size_t(1)) == -1
    assert oracle.orc_reduce_fold(0, 6, ptr(a), ptr(a), ctypes.c_size_t(1)) == -1
