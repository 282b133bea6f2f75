"""Subtask-reduction oracle pinned to the reference runtime's own fold.

oracle/_ref/libref_reduce.so holds pmReducer::ReduceMemories and
getBitwiseOperatableType (source/code/src/pmReducer.cpp:408-424, 590-700),
cut unchanged out of pmReducer.cpp by oracle/ref/extract_serial.py and
compiled against a stand-in declaration of the class, with the data-type
dispatch of pmReducer::ReduceExternalMemory (:502-540: INTS int, UNSIGNED_INTS
uint, LONGS long, UNSIGNED_LONGS ulong, FLOATS float, DOUBLES double).
tests/golden/reduce_golden.npz carries its outputs to machines without the
reference tree.  orc_reduce_fold (the oracle the device fold and the runtime
are checked against) must equal it bit for bit for every operation and type.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT, ptr
from test_reduce_oracle import DTYPES, values

GOLDEN = os.path.join(ROOT, "tests", "golden", "reduce_golden.npz")


def orc(oracle, op, code, a, b):
    r = a.copy()
    assert oracle.orc_reduce_fold(op, code, ptr(r), ptr(b), ctypes.c_size_t(a.size)) == 0
    return r


def same_bits(x, y):
    return x.dtype == y.dtype and x.tobytes() == y.tobytes()


@pytest.mark.parametrize("name", list(DTYPES))
def test_golden_reduce_every_operation(oracle, name):
    g = np.load(GOLDEN)
    code, _ = DTYPES[name]
    for op in range(10):
        a, b, want = g[f"{name}_op{op}_a"], g[f"{name}_op{op}_b"], g[f"{name}_op{op}_out"]
        assert same_bits(orc(oracle, op, code, a, b), want), (name, op)


@pytest.mark.parametrize("name", list(DTYPES))
def test_reference_reduce_memories_equals_oracle(oracle, name):
    path = os.path.join(ROOT, "oracle", "_ref", "libref_reduce.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    ref = ctypes.CDLL(path)
    code, dt = DTYPES[name]
    for op in range(10):
        a, b = values(dt, op, 4099, 3), values(dt, op, 4099, 4)
        want = a.copy()
        assert ref.ref_reduce_memories(op, code, ptr(want), ptr(b.copy()), ctypes.c_size_t(a.size)) == 0
        assert same_bits(orc(oracle, op, code, a, b), want), (name, op)
    # an operation outside the enumeration: the reference throws (pmFatalErrorException), the oracle refuses
    x = values(dt, 0, 8, 5)
    assert ref.ref_reduce_memories(10, code, ptr(x.copy()), ptr(x.copy()), ctypes.c_size_t(8)) == 2
    assert oracle.orc_reduce_fold(10, code, ptr(x.copy()), ptr(x.copy()), ctypes.c_size_t(8)) == -1
