"""CPU tests: PageRank oracles.  The fp32 push restatement is pinned to the
reference's own pageRank_cpu (oracle/_ref), and the FP64 pull oracle agrees
with both on the same graphs."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ptr


def random_graph(n, e, seed, skew=True):
    rng = np.random.default_rng(seed)
    if skew:  # a few hubs, like R-MAT
        src = (rng.pareto(1.2, e) * 3).astype(np.int64) % n
        dst = (rng.pareto(1.2, e) * 3).astype(np.int64) % n
        perm = rng.permutation(n)
        src, dst = perm[src], perm[dst]
    else:
        src, dst = rng.integers(0, n, e), rng.integers(0, n, e)
    return src.astype(np.uint32), dst.astype(np.uint32)


def csr_by_dst(src, dst, n):
    order = np.argsort(dst, kind="stable")
    col = src[order].astype(np.uint32)
    row_ptr = np.searchsorted(dst[order], np.arange(n + 1), side="left").astype(np.uint32)
    outdeg = np.bincount(src, minlength=n).astype(np.uint32)
    return row_ptr, col, outdeg


def out_lists(src, dst, n):
    order = np.argsort(src, kind="stable")
    out_ptr = np.searchsorted(src[order], np.arange(n + 1), side="left").astype(np.uint32)
    return out_ptr, dst[order].astype(np.uint32), src[order].astype(np.uint32)


def oracle_f64(oracle, row_ptr, col, outdeg, n, iters, init):
    out = np.zeros(n, np.float64)
    r0 = np.full(n, init, np.float32)
    oracle.orc_pagerank_f64(ptr(row_ptr), ptr(col), ptr(outdeg), n, iters, ctypes.c_double(0.85), ptr(r0), ptr(out))
    return out


def oracle_push(oracle, src, dst, n, outdeg, iters, init):
    out_ptr, out_dst, srt_src = out_lists(src, dst, n)
    out = np.zeros(n, np.float32)
    r0 = np.full(n, init, np.float32)
    oracle.orc_pagerank_push_f32(ptr(srt_src), ptr(out_dst), ctypes.c_uint64(src.size), n, ptr(outdeg), iters,
                                 ctypes.c_float(0.85), ptr(r0), ptr(out))
    return out


@pytest.mark.parametrize("n,e,iters", [(50, 300, 1), (1000, 20000, 2), (3000, 50000, 5)])
def test_push_oracle_matches_reference_callback(oracle, n, e, iters):
    import os

    from conftest import ROOT

    path = os.path.join(ROOT, "oracle", "_ref", "libref_pagerank.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built")
    ref = ctypes.CDLL(path)
    src, dst = random_graph(n, e, n + e)
    _, _, outdeg = csr_by_dst(src, dst, n)
    out_ptr, out_dst, _ = out_lists(src, dst, n)
    expect = np.zeros(n, np.float32)
    assert ref.ref_pagerank(ptr(out_ptr), ptr(out_dst), n, iters, ctypes.c_float(1.0 / n), ptr(expect)) == 0
    got = oracle_push(oracle, src, dst, n, outdeg, iters, 1.0 / n)
    assert np.array_equal(got, expect)  # same fp32 operations in the same order


def test_push_oracle_matches_golden_reference_ranks(oracle):
    """tests/golden/pagerank_golden.npz: the reference's pageRank_cpu ranks on
    two seeded hub-heavy graphs (written by tests/golden/make_golden.py), for
    machines without the reference tree.  Bit for bit."""
    import os

    from conftest import ROOT

    g = np.load(os.path.join(ROOT, "tests", "golden", "pagerank_golden.npz"))
    for idx in range(2):
        n, _, iters = (int(v) for v in g[f"g{idx}_meta"])
        src, dst = g[f"g{idx}_src"], g[f"g{idx}_dst"]
        _, _, outdeg = csr_by_dst(src, dst, n)
        got = oracle_push(oracle, src, dst, n, outdeg, iters, 1.0 / n)
        assert np.array_equal(got, g[f"g{idx}_rank"]), idx


def test_f64_oracle_close_to_push(oracle):
    n, e = 2000, 40000
    src, dst = random_graph(n, e, 3)
    row_ptr, col, outdeg = csr_by_dst(src, dst, n)
    r64 = oracle_f64(oracle, row_ptr, col, outdeg, n, 10, 1.0 / n)
    r32 = oracle_push(oracle, src, dst, n, outdeg, 10, 1.0 / n)
    assert np.abs(r64 - r32).sum() < 1e-5
    # no teleport: the total rank never grows
    assert r64.sum() <= 1.0 + 1e-12
