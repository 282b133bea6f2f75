"""Sentinel compression of reduction outputs (zero is the sentinel), in the
reference's compressed form: uint32 count, the non-zero elements, their
uint32 indices, in index order (pmCudaInterface.cu:380-472,
pmExecutionStub.cpp:3850-3950), compressed only when fewer than 40 % of the
elements are non-zero.  The device compressor is checked byte for byte
against that form built with numpy, and the host expander against the
original data."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ptr

TYPES = {0: np.int32, 1: np.uint32, 2: np.int64, 3: np.uint64, 4: np.float32, 5: np.float64}


def sparse(dtype, n, density, seed):
    rng = np.random.default_rng(seed)
    if np.issubdtype(dtype, np.floating):
        x = rng.uniform(-1000, 1000, n).astype(dtype)
    else:
        info = np.iinfo(dtype)
        x = rng.integers(max(info.min, -2**62), min(info.max, 2**62), n, dtype=np.int64).astype(dtype)
    x[rng.random(n) >= density] = 0
    return x


def packed_form(x):
    idx = np.flatnonzero(x).astype(np.uint32)
    return np.concatenate([np.array([idx.size], np.uint32).view(np.uint8), x[idx].view(np.uint8),
                           idx.view(np.uint8)])


@pytest.mark.parametrize("t", sorted(TYPES))
def test_expand_on_host(pmb, t):
    x = sparse(TYPES[t], 1000, 0.1, t)
    p = packed_form(x)
    out = np.full(x.size, 7, dtype=x.dtype)
    assert pmb.pmb_sentinel_expand(t, ptr(p), ptr(out), ctypes.c_size_t(x.nbytes)) == 0
    assert np.array_equal(out.view(np.uint8), x.view(np.uint8))


def test_decision_matches_the_reference_rule(pmb):
    n = 1000
    assert pmb.pmb_sentinel_compressed(0, ctypes.c_size_t(4 * n), 399) == 1
    assert pmb.pmb_sentinel_compressed(0, ctypes.c_size_t(4 * n), 400) == 0  # count < 0.4 x elements


@pytest.mark.gpu
@pytest.mark.parametrize("t", sorted(TYPES))
@pytest.mark.parametrize("n,density", [(1, 1.0), (4095, 0.1), (4097, 0.0), ((1 << 22) + 3, 0.1), (100000, 0.6)])
def test_device_compress_matches_reference_form(cuda, pmb, t, n, density):
    from unicorn_b200 import capi, ops

    x = sparse(TYPES[t], n, density, n + t)
    d = cuda.from_numpy(x.view(np.uint8).copy()).cuda()
    cap = pmb.pmb_sentinel_capacity_bytes(t, x.nbytes)
    scr = pmb.pmb_sentinel_scratch_bytes(t, x.nbytes)
    dst = ops._scratch(cap)
    sc = ops._scratch(scr)
    capi.check(pmb.pmb_sentinel_compress(t, d.data_ptr(), x.nbytes, dst.data_ptr(), cap, sc.data_ptr(), scr,
                                         cuda.cuda.current_stream().cuda_stream))
    cuda.cuda.synchronize()
    got = dst.cpu().numpy()
    count = int(got[:4].view(np.uint32)[0])
    assert count == np.count_nonzero(x)
    compressed = pmb.pmb_sentinel_compressed(t, ctypes.c_size_t(x.nbytes), count)
    assert compressed == (count < 0.4 * n)
    if compressed:
        p = packed_form(x)
        assert np.array_equal(got[:p.size], p)
        out = np.empty_like(x)
        assert pmb.pmb_sentinel_expand(t, ptr(got), ptr(out), ctypes.c_size_t(x.nbytes)) == 0
        assert np.array_equal(out.view(np.uint8), x.view(np.uint8))
