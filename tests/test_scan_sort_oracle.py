"""CPU tests: the prefixSum / radixSort oracles (restatements of
serialPrefixSum, prefixSum.cpp:47-53, and serialRadixSortRound,
radixSort.cpp:55-69) against independent numpy formulations."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ptr


def orc_scan(oracle, x):
    out = np.zeros(x.size, np.uint64)
    oracle.orc_prefix_sum_u32_u64(ptr(x), ptr(out), ctypes.c_size_t(x.size))
    return out


def orc_round(oracle, x, shift, bits):
    out = np.zeros_like(x)
    bins = np.zeros(1 << bits, np.uint32)
    oracle.orc_radix_round_u32(ptr(x), ptr(out), ctypes.c_size_t(x.size), shift, bits, ptr(bins))
    return out, bins


@pytest.mark.parametrize("n", [1, 2, 1000, 4097])
def test_scan_oracle(oracle, n):
    x = np.random.default_rng(n).integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(orc_scan(oracle, x), np.cumsum(x.astype(np.uint64)))


@pytest.mark.parametrize("bits", [4, 8])
def test_radix_round_is_stable_counting_sort(oracle, bits):
    x = np.random.default_rng(bits).integers(0, 2**32, size=5000, dtype=np.uint64).astype(np.uint32)
    for shift in range(0, 32, bits):
        d = (x >> shift) & ((1 << bits) - 1)
        out, bins = orc_round(oracle, x, shift, bits)
        assert np.array_equal(out, x[np.argsort(d, kind="stable")])
        assert np.array_equal(bins, np.bincount(d, minlength=1 << bits))


def test_radix_full_sort_oracle(oracle):
    x = np.random.default_rng(9).integers(0, 2**32, size=10000, dtype=np.uint64).astype(np.uint32)
    for bits in (4, 8):
        k = x.copy()
        tmp = np.zeros_like(k)
        oracle.orc_radix_sort_u32(ptr(k), ptr(tmp), ctypes.c_size_t(k.size), 0, 32, bits)
        assert np.array_equal(k, np.sort(x))
