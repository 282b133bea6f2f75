"""GPU test of the allocation-free scan entry point.

pmb_inclusive_scan_u32_u64_noalloc exists for callers that may not allocate
device memory (a pm:: subtask_gpu_custom callback must only enqueue work on
its stream; cudaMalloc would synchronise the device and stall the other
subtasks in flight) -- it keeps its scratch (tile counter, error word and
tile status words) in a fixed array inside libpmb.so.  Its results must equal the allocating entry point's bit for bit
(integer scan), on two calls in a row that reuse the shared array.  This file
is collected last so that a failure here comes after every other test has
run; it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_scan_matches_allocating_scan_twice(cuda, pmb):
    from unicorn_b200 import capi, ops

    stream = cuda.cuda.current_stream().cuda_stream
    for call, n in enumerate([(1 << 22) + 77, 1_000_003]):
        x = np.random.default_rng(40 + call).integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        d_in = cuda.from_numpy(x.view(np.int32)).cuda()
        expect, _ = ops.inclusive_scan_u32_u64(d_in)
        got = cuda.full((n,), -1, dtype=cuda.int64, device="cuda")
        capi.check(pmb.pmb_inclusive_scan_u32_u64_noalloc(d_in.data_ptr(), got.data_ptr(), n, stream))
        cuda.cuda.synchronize()
        assert noalloc_error(pmb) == 0
        assert cuda.equal(got, expect), f"call {call}: differs from pmb_inclusive_scan_u32_u64"
        assert np.array_equal(got.cpu().numpy().view(np.uint64), np.cumsum(x, dtype=np.uint64))


def noalloc_error(pmb) -> int:
    from unicorn_b200 import capi

    err = ctypes.c_uint32(0xFFFFFFFF)
    capi.check(pmb.pmb_scan_noalloc_error(ctypes.byref(err)))
    return int(err.value)


@pytest.mark.parametrize("n", [1 << 28, (1 << 29) + 4097])
def test_noalloc_scan_full_size(cuda, pmb, n):
    """The prefix-sum configuration (2^28 keys, sorted first) and a ragged
    2^29 + 4097 random input: equal to the allocating entry point, exact by
    consecutive differences, error word clear."""
    from unicorn_b200 import capi, ops

    g = cuda.Generator(device="cuda")
    g.manual_seed(n)
    d_in = cuda.randint(-(2**31), 2**31, (n,), dtype=cuda.int32, device="cuda", generator=g)
    if n == 1 << 28:
        ops.radix_sort_u32(d_in)
    stream = cuda.cuda.current_stream().cuda_stream
    got = cuda.full((n,), -1, dtype=cuda.int64, device="cuda")
    capi.check(pmb.pmb_inclusive_scan_u32_u64_noalloc(d_in.data_ptr(), got.data_ptr(), n, stream))
    cuda.cuda.synchronize()
    assert noalloc_error(pmb) == 0
    x = d_in.to(cuda.int64) & 0xFFFFFFFF
    assert int(got[0]) == int(x[0]) and cuda.equal(got[1:] - got[:-1], x[1:])
    del x
    expect, _ = ops.inclusive_scan_u32_u64(d_in)
    cuda.cuda.synchronize()
    assert cuda.equal(got, expect)


def test_noalloc_scan_rejects_inputs_beyond_its_fixed_scratch(pmb):
    from unicorn_b200 import capi

    st = pmb.pmb_inclusive_scan_u32_u64_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16),
                                                capi.PMB_SCAN_NOALLOC_MAX_ELEMS + 1, None)
    assert st == capi.PMB_BEYOND_LIMITS
    assert b"fixed scratch limit" in pmb.pmb_last_error()
