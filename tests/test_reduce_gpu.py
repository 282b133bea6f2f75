"""GPU parity of the device subtask reduction (pmb_reduce_elementwise) with
the oracle's restatement of pmReducer::ReduceMemories: every operation on
every data type, bit-exact (sources folded in order, so float sums match the
sequential host fold), one- and multi-launch source counts, vector and
unaligned (scalar) paths, folding into an existing destination."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from test_reduce_oracle import DTYPES, oracle_fold, values

pytestmark = pytest.mark.gpu


def run_device(cuda, op, type_code, srcs, count, dst0=None, offset=0):
    """Fold on the device; `offset` elements shift every pointer off 16-byte alignment."""
    from unicorn_b200 import ops

    dt = srcs[0].dtype
    d_srcs = [cuda.from_numpy(np.concatenate([np.zeros(offset, dt), s]).view(np.uint8)).cuda() for s in srcs]
    dst_host = np.concatenate([np.zeros(offset, dt), dst0 if dst0 is not None else np.zeros(count, dt)])
    d_dst = cuda.from_numpy(dst_host.view(np.uint8).copy()).cuda()
    es = dt.itemsize
    views = [t[offset * es:] for t in d_srcs]
    ops.reduce_elementwise(op, type_code, d_dst[offset * es:], views, count, init_from_first=dst0 is None)
    cuda.cuda.synchronize()
    return d_dst.cpu().numpy().view(dt)[offset:]


@pytest.mark.parametrize("type_name", list(DTYPES))
@pytest.mark.parametrize("op", range(10))
def test_every_operation_matches_oracle(cuda, oracle, op, type_name):
    type_code, dt = DTYPES[type_name]
    count = (1 << 16) + 5
    srcs = [values(dt, op, count, seed) for seed in range(7)]
    want = oracle_fold(oracle, op, type_code, srcs)
    got = run_device(cuda, op, type_code, srcs, count)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))


@pytest.mark.parametrize("nsrc,count,offset", [(1, 1, 0), (2, 3, 1), (5, 1000, 0), (5, 1001, 1), (128, 4099, 0),
                                               (129, 4099, 0), (300, 777, 1), (9, (1 << 22) + 7, 0)])
def test_source_counts_and_alignment(cuda, oracle, nsrc, count, offset):
    type_code, dt = DTYPES["float32"]
    srcs = [values(dt, 0, count, seed) for seed in range(nsrc)]
    want = oracle_fold(oracle, 0, type_code, srcs)
    got = run_device(cuda, 0, type_code, srcs, count, offset=offset)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))


@pytest.mark.parametrize("type_name", ["int64", "float64"])
def test_fold_into_existing_destination(cuda, oracle, type_name):
    type_code, dt = DTYPES[type_name]
    count = 12345
    dst0 = values(dt, 2, count, 99)
    srcs = [values(dt, 2, count, seed) for seed in range(3)]
    want = oracle_fold(oracle, 2, type_code, [dst0] + srcs)
    got = run_device(cuda, 2, type_code, srcs, count, dst0=dst0)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))


def test_rejects_bad_arguments_before_launch(cuda):
    """Unknown operations / types and misaligned pointers are refused on the
    host; nothing is launched."""
    from unicorn_b200 import capi

    L = capi.lib()
    d = cuda.zeros(64, dtype=cuda.uint8, device="cuda")
    p = (ctypes.c_void_p * 1)(d.data_ptr())
    arr = ctypes.cast(p, ctypes.c_void_p)
    s = cuda.cuda.current_stream().cuda_stream
    assert L.pmb_reduce_elementwise(10, 0, d.data_ptr(), arr, 1, 4, 1, s) == capi.PMB_INVALID_INDEX
    assert L.pmb_reduce_elementwise(0, 6, d.data_ptr(), arr, 1, 4, 1, s) == capi.PMB_INVALID_INDEX
    assert L.pmb_reduce_elementwise(0, 2, d.data_ptr() + 4, arr, 1, 4, 1, s) == capi.PMB_INVALID_INDEX
    assert L.pmb_reduce_elementwise(0, 0, d.data_ptr(), arr, 0, 4, 1, s) == capi.PMB_INVALID_INDEX
    cuda.cuda.synchronize()
