"""GPU parity tests of the chunked reduce-then-scan and the onesweep radix sort.

Integer results must be bit-exact against the oracles (restatements of the
reference's serialPrefixSum / serialRadixSortRound); every run also checks
that no look-back wait gave up (scratch error word 0).
"""
from __future__ import annotations

import numpy as np
import pytest

from test_scan_sort_oracle import orc_round, orc_scan

pytestmark = pytest.mark.gpu


def keys(n, seed, kind="uniform"):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        return rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    if kind == "equal":
        return np.full(n, 0xDEADBEEF, np.uint32)
    if kind == "sorted":
        return np.sort(keys(n, seed))
    if kind == "reverse":
        return np.sort(keys(n, seed))[::-1].copy()
    if kind == "few":
        return rng.integers(0, 3, size=n, dtype=np.uint32) << np.uint32(24)
    raise ValueError(kind)


def to_dev(cuda, x):
    return cuda.from_numpy(x.view(np.int32)).cuda()


@pytest.mark.parametrize("n", [1, 3, 4, 5, 4095, 4096, 4097, 8192 + 17, 32768 + 1, 1 << 20, (1 << 22) + 3,
                               (1 << 23) + 5, 3 * (1 << 23) + 12345])
def test_scan_matches_oracle(cuda, oracle, n):
    from unicorn_b200 import ops

    x = keys(n, n)
    out, scratch = ops.inclusive_scan_u32_u64(to_dev(cuda, x))
    cuda.cuda.synchronize()
    got = out.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, orc_scan(oracle, x))
    assert ops.scratch_error(scratch) == 0


def test_scan_carries_of_maximal_values(cuda):
    """All keys 2^32-1 across a chunk boundary: carries and segment sums
    need their full 64 bits."""
    from unicorn_b200 import ops

    n = (1 << 23) + 4099
    x = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
    out, scratch = ops.inclusive_scan_u32_u64(to_dev(cuda, x))
    cuda.cuda.synchronize()
    got = out.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0xFFFFFFFF))


def test_scan_repeated_calls_reuse_scratch(cuda):
    from unicorn_b200 import ops

    x = keys(100003, 1)
    d = to_dev(cuda, x)
    out, scratch = ops.inclusive_scan_u32_u64(d)
    for _ in range(3):
        out2, scratch = ops.inclusive_scan_u32_u64(d, scratch=scratch)
    cuda.cuda.synchronize()
    assert np.array_equal(out2.cpu().numpy().view(np.uint64), np.cumsum(x.astype(np.uint64)))


@pytest.mark.parametrize("bits", [8, 4])
@pytest.mark.parametrize("n", [1, 7, 4096, 4097, 100000, (1 << 21) + 5])
def test_radix_sort_full(cuda, bits, n):
    from unicorn_b200 import ops

    x = keys(n, n + bits)
    d = to_dev(cuda, x)
    _, scratch = ops.radix_sort_u32(d, 0, 32, bits)
    cuda.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), np.sort(x))
    assert ops.scratch_error(scratch) == 0


@pytest.mark.parametrize("kind", ["equal", "sorted", "reverse", "few"])
def test_radix_sort_edge_distributions(cuda, kind):
    from unicorn_b200 import ops

    x = keys(300001, 5, kind)
    d = to_dev(cuda, x)
    ops.radix_sort_u32(d)
    cuda.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), np.sort(x))


@pytest.mark.parametrize("bits", [4, 8])
def test_single_round_matches_reference_round(cuda, oracle, bits):
    """One pass == one reference round (per-subtask counting sort + ordered
    redistribution), including the stable order of equal digits."""
    from unicorn_b200 import ops

    x = keys(123457, 77)
    for shift in range(0, 32, bits):
        d = to_dev(cuda, x)
        ops.radix_sort_u32(d, shift, shift + bits, bits)
        cuda.cuda.synchronize()
        expect, _ = orc_round(oracle, x, shift, bits)
        assert np.array_equal(d.cpu().numpy().view(np.uint32), expect), shift


def scan_is_exact(cuda, d_in, out) -> bool:
    """Size-independent check of an inclusive scan on the device: the first
    sum is the first key and consecutive sums differ by exactly the next key
    (64-bit sums of n <= 2^30 keys stay below 2^62, so int64 holds them)."""
    x = d_in.to(cuda.int64) & 0xFFFFFFFF
    if out.numel() != x.numel() or int(out[0]) != int(x[0]):
        return False
    return bool(cuda.equal(out[1:] - out[:-1], x[1:]))


def test_sort_then_scan_full_configuration(cuda):
    """2^28 uint32 keys (seed 2): 8-bit LSD sort, then inclusive uint64 scan."""
    from unicorn_b200 import ops

    n = 1 << 28
    x = keys(n, 2)
    d = to_dev(cuda, x)
    _, s1 = ops.radix_sort_u32(d)
    out, s2 = ops.inclusive_scan_u32_u64(d)
    cuda.cuda.synchronize()
    assert ops.scratch_error(s1) == 0 and ops.scratch_error(s2) == 0
    ref_sorted = np.sort(x)
    assert np.array_equal(d.cpu().numpy().view(np.uint32), ref_sorted)
    del x
    assert np.array_equal(out.cpu().numpy().view(np.uint64), np.cumsum(ref_sorted, dtype=np.uint64))


@pytest.mark.parametrize("n,where", [(1 << 28, "created stream"), (1 << 28, "default stream"),
                                     ((1 << 28) + 12345, "default stream"), (1 << 29, "created stream")])
def test_scan_full_size(cuda, n, where):
    """2^28 and 2^29 random keys (16 and 32 blocks of 2^24), alone on a
    created stream or the default stream, and a ragged 2^28 + 12345."""
    from unicorn_b200 import ops

    g = cuda.Generator(device="cuda")
    g.manual_seed(n)
    d = cuda.randint(-(2**31), 2**31, (n,), dtype=cuda.int32, device="cuda", generator=g)
    if where == "created stream":
        s = cuda.cuda.Stream()
        s.wait_stream(cuda.cuda.current_stream())
        with cuda.cuda.stream(s):
            out, scratch = ops.inclusive_scan_u32_u64(d, stream=s)
        s.synchronize()
    else:
        out, scratch = ops.inclusive_scan_u32_u64(d)
        cuda.cuda.synchronize()
    assert ops.scratch_error(scratch) == 0
    assert scan_is_exact(cuda, d, out)


def test_scan_sorted_run_twice_same_scratch(cuda):
    """Two scans of the full configuration back to back on one scratch buffer
    (the second must clear what the first left behind)."""
    from unicorn_b200 import ops

    n = 1 << 28
    g = cuda.Generator(device="cuda")
    g.manual_seed(2)
    d = cuda.randint(-(2**31), 2**31, (n,), dtype=cuda.int32, device="cuda", generator=g)
    ops.radix_sort_u32(d)
    out, scratch = ops.inclusive_scan_u32_u64(d)
    out2, scratch = ops.inclusive_scan_u32_u64(d, scratch=scratch)
    cuda.cuda.synchronize()
    assert ops.scratch_error(scratch) == 0
    assert scan_is_exact(cuda, d, out2) and cuda.equal(out, out2)


def test_scan_after_producer_on_same_stream(cuda):
    """The chunk launches overlap by programmatic dependent launch; the first
    one must wait for a kernel that writes the input earlier on the stream."""
    from unicorn_b200 import ops

    n = 3 * (1 << 24) + 77
    x = keys(n, 9)
    src = to_dev(cuda, x)
    d = cuda.zeros_like(src)
    s = cuda.cuda.Stream()
    with cuda.cuda.stream(s):
        d.copy_(src)
        out, scratch = ops.inclusive_scan_u32_u64(d, stream=s)
        d.zero_()                        # queued behind the scan: must not change its result
    s.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), np.cumsum(x.astype(np.uint64)))
