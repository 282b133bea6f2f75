"""prefixSum and radixSort oracles pinned to the reference's serial functions.

oracle/_ref/libref_scan_sort.so holds the reference's serialPrefixSum
(prefixSum.cpp:47-53) and serialRadixSortRound / serialLsbRadixSortRound /
serialLsbRadixSort (radixSort.cpp:46-114), cut unchanged out of those files
by oracle/ref/extract_serial.py (the files' task code does not compile).
tests/golden/scan_sort_golden.npz carries their outputs to machines without
the reference tree.  Bit-exact throughout:

* the reference scans int32; orc_prefix_sum_u32_u64 (the u32 -> u64 form the
  kernels compute) equals it wherever int32 does not overflow;
* the reference sorts in BITS_PER_ROUND (4) bit digits; orc_radix_round_u32
  equals each of its rounds (output order and digit counts), and
  orc_radix_sort_u32 equals its full sort with 4- and with 8-bit digits.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT, ptr

GOLDEN = os.path.join(ROOT, "tests", "golden", "scan_sort_golden.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def ref():
    path = os.path.join(ROOT, "oracle", "_ref", "libref_scan_sort.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    return ctypes.CDLL(path)


def orc_scan(oracle, x):
    xu = np.ascontiguousarray(x, dtype=np.uint32)
    out = np.zeros(xu.size, np.uint64)
    oracle.orc_prefix_sum_u32_u64(ptr(xu), ptr(out), ctypes.c_size_t(xu.size))
    return out


def orc_round(oracle, keys, shift, bits):
    out = np.zeros_like(keys)
    bins = np.zeros(1 << bits, np.uint32)
    oracle.orc_radix_round_u32(ptr(keys), ptr(out), ctypes.c_size_t(keys.size), shift, bits, ptr(bins))
    return out, bins


def orc_sort(oracle, keys, bits):
    k = keys.copy()
    tmp = np.empty_like(k)
    oracle.orc_radix_sort_u32(ptr(k), ptr(tmp), ctypes.c_size_t(k.size), 0, 32, bits)
    return k


# ---------------------------------------------------------------- golden


def test_golden_scan(oracle, golden):
    x, y = golden["scan_in"], golden["scan_out"]
    assert np.array_equal(orc_scan(oracle, x), y.astype(np.uint64))


def test_golden_rounds_and_sort(oracle, golden):
    bits, rounds = (int(v) for v in golden["sort_meta"])
    keys = golden["sort_in"]
    for r in range(rounds):
        out, bins = orc_round(oracle, keys, r * bits, bits)
        assert np.array_equal(out, golden[f"round{r}_out"]), r
        assert np.array_equal(bins.astype(np.int32), golden[f"round{r}_bins"]), r
    assert np.array_equal(orc_sort(oracle, keys, bits), golden["sort_out"])
    assert np.array_equal(orc_sort(oracle, keys, 8), golden["sort_out"])


# ---------------------------------------------------------------- reference tree


@pytest.mark.parametrize("n,hi", [(1, 5), (2, 1 << 20), (100_000, 1 << 12), (1 << 20, 1 << 11)])
def test_reference_scan_equals_oracle(oracle, ref, n, hi):
    x = np.random.default_rng(n).integers(0, hi, n, dtype=np.int32)
    y = np.zeros_like(x)
    ref.ref_serial_prefix_sum_i32(ptr(x), ptr(y), ctypes.c_uint(n))
    assert np.array_equal(orc_scan(oracle, x), y.astype(np.uint64))


@pytest.mark.parametrize("kind", ["uniform", "few", "sorted", "reverse", "equal"])
def test_reference_radix_equals_oracle(oracle, ref, kind):
    rng = np.random.default_rng(7)
    n = 1 << 18
    keys = {"uniform": rng.integers(0, 2**32, n, dtype=np.uint32),
            "few": rng.integers(0, 4, n, dtype=np.uint32) * np.uint32(0x11111111),
            "sorted": np.sort(rng.integers(0, 2**32, n, dtype=np.uint32)),
            "reverse": np.sort(rng.integers(0, 2**32, n, dtype=np.uint32))[::-1].copy(),
            "equal": np.full(n, 0xDEADBEEF, np.uint32)}[kind]
    bits, rounds = ref.ref_radix_bits_per_round(), ref.ref_radix_total_rounds()
    assert (bits, rounds) == (4, 8)
    for r in range(rounds):
        want = np.zeros_like(keys)
        wbins = np.zeros(1 << bits, np.int32)
        ref.ref_serial_lsb_radix_round_u32(ptr(keys), ptr(want), ctypes.c_uint(n), r, ptr(wbins))
        got, gbins = orc_round(oracle, keys, r * bits, bits)
        assert np.array_equal(got, want) and np.array_equal(gbins.astype(np.int32), wbins), r
    want = np.zeros_like(keys)
    ref.ref_serial_lsb_radix_sort_u32(ptr(keys), ptr(want), ctypes.c_uint(n), rounds)
    assert np.array_equal(orc_sort(oracle, keys, 4), want)
    assert np.array_equal(orc_sort(oracle, keys, 8), want)
