"""The reference pageRank app's own input format and decomposition.

* The unchanged app (pageRank.cpp + commonAPI.cpp from the reference tree,
  oracle/_ref/pageRank_b200.exe) reads a web dump written by tests/webdump.py
  and runs its tasks through this runtime: 4 subtasks of page ranges, each
  writing its own copy of the whole rank array, folded by the app's
  REDUCE_ADD callback -- on the host in parallel mode 1 (its pageRank_cpu),
  on the device in mode 2 (pageRank_cudaLaunchFunc from
  libpmb_app_pageRank.so).  The app compares with its own serial run.  Its
  skewed graph gives ranks in the hundreds, so a lost subtask copy fails the
  app's |serial - parallel| < 1 check.
* pmb_webdump_push (the reference's push step) against the oracle's fp32 push
  (pageRank_cpu restated), relative 2e-4 (the device adds in no fixed order;
  hub pages sum thousands of fp32 terms).
* pmb_csr_from_webdump against pmb_csr_by_destination of the same edges:
  identical arrays; out-of-range targets and over-long counts flagged.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, ptr
from webdump import edges_of, make_dump, write_webdump

APP = os.path.join(ROOT, "oracle", "_ref", "pageRank_b200.exe")


def app_or_skip():
    if not os.path.exists(APP):
        pytest.skip("oracle/_ref/pageRank_b200.exe not built (reference tree absent)")
    return APP


@pytest.fixture(scope="module")
def dump_dir(tmp_path_factory):
    base = str(tmp_path_factory.mktemp("web_dump"))
    write_webdump(base, make_dump(8 * 4096, 24, seed=11, skew=3.0), 4096)
    return base


def run(cmd, timeout=600):
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    return p.returncode, p.stdout + p.stderr


def test_reference_app_cpu_with_host_reduction(dump_dir):
    rc, out = run([app_or_skip(), "1", "1", "0", dump_dir])
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out


@pytest.mark.gpu
def test_reference_app_gpu_with_device_reduction(dump_dir):
    rc, out = run([app_or_skip(), "1", "2", "0", dump_dir])
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out


@pytest.mark.gpu
def test_reference_app_single_gpu(dump_dir):
    """Run mode 4: the app's serial run, then singleGpuPageRank (CSR built from
    the whole dump, pull iterations), compared by the app."""
    rc, out = run([app_or_skip(), "4", "2", "0", dump_dir])
    assert rc == 0 and "Single GPU Task's Sequential Comparison Test Passed" in out, out


def _dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("n,maxo,with_rank", [(1, 1, False), (1000, 7, True), (65536, 40, False),
                                              (300001, 13, True)])
def test_webdump_push_matches_oracle(cuda, oracle, n, maxo, with_rank):
    from unicorn_b200 import capi

    L = capi.lib()
    dump = make_dump(n, maxo, seed=n, skew=2.0)
    rng = np.random.default_rng(n)
    rank = (rng.random(n) + 0.5).astype(np.float32) if with_rank else np.ones(n, np.float32)
    d_dump = _dev(cuda, dump)
    d_rank = _dev(cuda, rank)
    d_out = cuda.full((n,), 7.0, dtype=cuda.float32, device="cuda")
    d_err = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    st = L.pmb_webdump_push(d_dump.data_ptr(), n, maxo, d_rank.data_ptr() if with_rank else None, 1.0, 0.85,
                            d_out.data_ptr(), n, d_err.data_ptr(), cuda.cuda.current_stream().cuda_stream)
    assert st == 0
    got = d_out.cpu().numpy()
    src, dst = edges_of(dump)
    outdeg = dump[:, 0].copy()
    want = np.zeros(n, np.float32)
    oracle.orc_pagerank_push_f32(ptr(src), ptr(dst), ctypes.c_uint64(src.size), n, ptr(outdeg), 1,
                                 ctypes.c_float(0.85), ptr(rank), ptr(want))
    assert int(d_err.cpu()[0]) == 0
    np.testing.assert_allclose(got, want, rtol=2e-4, atol=1e-6)


@pytest.mark.gpu
def test_webdump_push_flags_bad_pages(cuda):
    from unicorn_b200 import capi

    L = capi.lib()
    dump = make_dump(100, 4, seed=3)
    dump[5, 0], dump[5, 1:] = 2, [0, 101, 0, 0]   # both targets out of range: skipped
    dump[9, 0] = 9                                 # count above the 4 slots: clamped
    d_dump = _dev(cuda, dump)
    d_out = cuda.zeros(100, dtype=cuda.float32, device="cuda")
    d_err = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    assert L.pmb_webdump_push(d_dump.data_ptr(), 100, 4, None, 1.0, 0.85, d_out.data_ptr(), 100, d_err.data_ptr(),
                              cuda.cuda.current_stream().cuda_stream) == 0
    assert int(d_err.cpu()[0]) & 2
    assert np.isfinite(d_out.cpu().numpy()).all()


@pytest.mark.gpu
@pytest.mark.parametrize("n,maxo", [(1, 3), (777, 9), (1 << 17, 30)])
def test_csr_from_webdump_equals_edge_builder(cuda, n, maxo):
    from unicorn_b200 import capi, ops

    L = capi.lib()
    dump = make_dump(n, maxo, seed=n + 1, skew=2.0)
    src, dst = edges_of(dump)
    E = src.size
    s = cuda.cuda.current_stream().cuda_stream
    outs = []
    for kind in ("dump", "edges"):
        row_ptr = cuda.zeros(n + 1, dtype=cuda.int32, device="cuda")
        col = cuda.zeros(max(E, 1), dtype=cuda.int32, device="cuda")
        deg = cuda.zeros(n, dtype=cuda.int32, device="cuda")
        if kind == "dump":
            sc = ops._scratch(L.pmb_webdump_csr_scratch_bytes(n, n, E))
            d_dump = _dev(cuda, dump)
            assert L.pmb_csr_from_webdump(d_dump.data_ptr(), n, maxo, n, E, row_ptr.data_ptr(), col.data_ptr(),
                                          deg.data_ptr(), sc.data_ptr(), sc.numel(), s) == 0
        else:
            sc = ops._scratch(L.pmb_csr_scratch_bytes(n, E))
            d_src, d_dst = _dev(cuda, src), _dev(cuda, dst)
            assert L.pmb_csr_by_destination(d_src.data_ptr(), d_dst.data_ptr(), n, E, row_ptr.data_ptr(),
                                            col.data_ptr(), deg.data_ptr(), sc.data_ptr(), sc.numel(), s) == 0
        cuda.cuda.synchronize()
        assert ops.scratch_error(sc) == 0
        outs.append((row_ptr.cpu().numpy(), col.cpu().numpy()[:E], deg.cpu().numpy()))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    assert np.array_equal(outs[0][2].view(np.uint32), dump[:, 0])


@pytest.mark.gpu
def test_csr_from_webdump_flags_bad_pages(cuda):
    from unicorn_b200 import capi, ops

    L = capi.lib()
    n, maxo = 50, 4
    dump = make_dump(n, maxo, seed=8)
    dump[3, 0], dump[3, 1] = 1, 0      # target 0 (outside [1, n])
    dump[7, 0], dump[7, 1:] = 6, [1, 2, 3, 4]   # count above the slots: clamped to 4
    E = int(np.minimum(dump[:, 0], maxo).sum())
    row_ptr = cuda.zeros(n + 1, dtype=cuda.int32, device="cuda")
    col = cuda.zeros(E, dtype=cuda.int32, device="cuda")
    deg = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    sc = ops._scratch(L.pmb_webdump_csr_scratch_bytes(n, n, E))
    d_dump = _dev(cuda, dump)
    assert L.pmb_csr_from_webdump(d_dump.data_ptr(), n, maxo, n, E, row_ptr.data_ptr(), col.data_ptr(),
                                  deg.data_ptr(), sc.data_ptr(), sc.numel(), cuda.cuda.current_stream().cuda_stream) == 0
    err = ops.scratch_error(sc)
    assert err & 2 and err & 4
    assert int(row_ptr.cpu()[n]) == E - 1   # the bad edge is dropped
