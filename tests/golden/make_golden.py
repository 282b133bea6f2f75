"""Generate golden fixtures from the reference's own CPU code.

* imageFilter: runs the reference's imageFilterDataDistribution +
  imageFilter_cpu (compiled unchanged from
  testSuite/imageFiltering/source/code/src/imageFiltering.cpp into
  oracle/_ref/libref_imgf.so by oracle/ref/Makefile) on small seeded inputs and
  stores inputs, filters and outputs in imgf_golden.npz, plus the reference's
  subscription geometry for a few image shapes in imgf_subscriptions.json.
* matrixMultiplyBlas and luDecomposition: runs the reference's
  matrixMultiplyDataDistribution + matrixMultiply_cpu and serialLUDecomposition
  (matrixMultiplyBlas.cpp, luDecomposition.cpp, compiled unchanged into
  oracle/_ref/libref_mm.so and libref_lu.so over a CBLAS shim on numpy's
  OpenBLAS) on small seeded inputs, and records the GEMM subscription geometry
  of the 1024 (blocks of 256) and 4096 (blocks of 2048) tasks: blas_golden.npz.
* prefixSum and radixSort: runs the reference's serialPrefixSum and
  serialLsbRadixSort / serialLsbRadixSortRound (cut unchanged out of
  prefixSum.cpp and radixSort.cpp by oracle/ref/extract_serial.py into
  oracle/_ref/libref_scan_sort.so) on seeded inputs: scan_sort_golden.npz.
* subtask reduction: runs the reference runtime's pmReducer::ReduceMemories
  (cut unchanged out of pmReducer.cpp into oracle/_ref/libref_reduce.so) for
  every operation and data type on the inputs tests/test_reduce_oracle.py
  generates: reduce_golden.npz.
* pageRank: runs the reference's pageRank_cpu (pageRank.cpp compiled unchanged
  into oracle/_ref/libref_pagerank.so) on seeded hub-heavy graphs from
  tests/test_pagerank_oracle.py: pagerank_golden.npz.

Usage (in a tree where the reference is available):
    make -C oracle/ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# (W, H, R, seed): odd sizes, heavy clamping (R larger than the image), and a
# width that spans two reference subtasks (TILE_DIM 2048).
CASES = [(37, 35, 1, 11), (67, 41, 2, 12), (130, 70, 3, 13), (20, 20, 15, 14), (5, 3, 2, 15),
         (2050, 5, 2, 16)]
SUB_SHAPES = [(8192, 8192, 2), (2100, 2050, 3), (4096, 2049, 1)]


def main() -> None:
    ref = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_imgf.so"))
    ref.ref_imgf_subtask_count.restype = ctypes.c_ulong
    P = ctypes.c_void_p
    out = {}
    for idx, (W, H, R, seed) in enumerate(CASES):
        rng = np.random.default_rng(seed)
        img = rng.integers(0, 256, size=H * W * 3, dtype=np.uint8)
        f = np.zeros((32, 32), np.int8)
        f[: 2 * R + 1, : 2 * R + 1] = rng.integers(-128, 128, size=(2 * R + 1, 2 * R + 1))
        res = np.zeros_like(img)
        st = ref.ref_imgf_task(img.ctypes.data_as(P), res.ctypes.data_as(P), W, H, R,
                               f.ctypes.data_as(P), 1, 0)
        assert st == 0, st
        out[f"c{idx}_meta"] = np.array([W, H, R, seed], np.int64)
        out[f"c{idx}_in"] = img
        out[f"c{idx}_filter"] = f
        out[f"c{idx}_out"] = res
    np.savez_compressed(os.path.join(HERE, "imgf_golden.npz"), **out)

    subs = []
    buf = (ctypes.c_ulonglong * 8)()
    for (W, H, R) in SUB_SHAPES:
        n = ref.ref_imgf_subtask_count(W, H)
        rows = []
        for sid in range(n):
            assert ref.ref_imgf_subscriptions(W, H, R, ctypes.c_ulong(sid), buf) == 0
            rows.append([int(x) for x in buf])
        subs.append({"W": W, "H": H, "R": R, "tile_dim": ref.ref_imgf_tile_dim(), "subtasks": rows})
    with open(os.path.join(HERE, "imgf_subscriptions.json"), "w") as fh:
        json.dump(subs, fh)


# GEMM (n, block, seed) and LU (n, ld, seed) cases of blas_golden.npz.
MM_CASES = [(64, 32, 21), (96, 48, 22)]
LU_CASES = [(7, 7, 23), (48, 50, 24)]
MM_SUB_SHAPES = [(1024, 256), (4096, 2048)]


def main_blas() -> None:
    P = ctypes.c_void_p
    mm = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_mm.so"))
    lu = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_lu.so"))
    out = {}
    for idx, (n, block, seed) in enumerate(MM_CASES):
        rng = np.random.default_rng(seed)
        a = rng.uniform(-1, 1, (n, n)).astype(np.float32)
        b = rng.uniform(-1, 1, (n, n)).astype(np.float32)
        c = np.zeros_like(a)
        st = mm.ref_mm_task(a.ctypes.data_as(P), b.ctypes.data_as(P), c.ctypes.data_as(P), ctypes.c_ulong(n),
                            ctypes.c_ulong(block))
        assert st == 0, st
        out[f"mm{idx}_meta"] = np.array([n, block, seed], np.int64)
        out[f"mm{idx}_a"], out[f"mm{idx}_b"], out[f"mm{idx}_c"] = a, b, c
    for idx, (n, ld, seed) in enumerate(LU_CASES):
        rng = np.random.default_rng(seed)
        a = rng.uniform(-1, 1, (n, ld)).astype(np.float32)  # row k of this array = column k (column-major)
        a[np.arange(n), np.arange(n)] += n
        r = a.copy()
        assert lu.ref_lu_serial(r.ctypes.data_as(P), ctypes.c_ulong(n), ctypes.c_ulong(ld)) == 0
        out[f"lu{idx}_meta"] = np.array([n, ld, seed], np.int64)
        out[f"lu{idx}_in"], out[f"lu{idx}_out"] = a, r
    buf = (ctypes.c_ulonglong * 15)()
    for idx, (n, block) in enumerate(MM_SUB_SHAPES):
        rows = []
        for sid in range((n // block) ** 2):
            assert mm.ref_mm_subscriptions(ctypes.c_ulong(n), ctypes.c_ulong(block), ctypes.c_ulong(sid), buf) == 0
            rows.append([int(x) for x in buf])
        out[f"mmsub{idx}_meta"] = np.array([n, block], np.int64)
        out[f"mmsub{idx}"] = np.array(rows, np.uint64)
    np.savez_compressed(os.path.join(HERE, "blas_golden.npz"), **out)


def main_scan_sort() -> None:
    P = ctypes.c_void_p
    ref = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_scan_sort.so"))
    out = {}
    rng = np.random.default_rng(31)
    # int32 scan (the reference's type) of values that cannot overflow it
    x = rng.integers(0, 1 << 20, 1000, dtype=np.int32)
    y = np.zeros_like(x)
    ref.ref_serial_prefix_sum_i32(x.ctypes.data_as(P), y.ctypes.data_as(P), ctypes.c_uint(x.size))
    out["scan_in"], out["scan_out"] = x, y
    # full LSD sort (BITS_PER_ROUND-bit digits, TOTAL_ROUNDS rounds) and each single round
    rng = np.random.default_rng(32)
    keys = np.concatenate([rng.integers(0, 2**32, 2500, dtype=np.uint32),
                           rng.integers(0, 8, 500, dtype=np.uint32) * np.uint32(0x10203041)])
    rounds = ref.ref_radix_total_rounds()
    srt = np.zeros_like(keys)
    ref.ref_serial_lsb_radix_sort_u32(keys.ctypes.data_as(P), srt.ctypes.data_as(P), ctypes.c_uint(keys.size),
                                      rounds)
    out["sort_meta"] = np.array([ref.ref_radix_bits_per_round(), rounds], np.int64)
    out["sort_in"], out["sort_out"] = keys, srt
    for r in range(rounds):
        o = np.zeros_like(keys)
        bins = np.zeros(1 << ref.ref_radix_bits_per_round(), np.int32)
        ref.ref_serial_lsb_radix_round_u32(keys.ctypes.data_as(P), o.ctypes.data_as(P), ctypes.c_uint(keys.size),
                                           r, bins.ctypes.data_as(P))
        out[f"round{r}_out"], out[f"round{r}_bins"] = o, bins
    np.savez_compressed(os.path.join(HERE, "scan_sort_golden.npz"), **out)


def main_reduce() -> None:
    import sys

    sys.path.insert(0, os.path.dirname(HERE))
    from test_reduce_oracle import DTYPES, values

    P = ctypes.c_void_p
    ref = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_reduce.so"))
    out = {}
    for name, (code, dt) in DTYPES.items():
        for op in range(10):
            a, b = values(dt, op, 33, 1), values(dt, op, 33, 2)
            r = a.copy()
            assert ref.ref_reduce_memories(op, code, r.ctypes.data_as(P), b.copy().ctypes.data_as(P),
                                           ctypes.c_size_t(a.size)) == 0
            out[f"{name}_op{op}_a"], out[f"{name}_op{op}_b"], out[f"{name}_op{op}_out"] = a, b, r
    np.savez_compressed(os.path.join(HERE, "reduce_golden.npz"), **out)


def main_pagerank() -> None:
    import sys

    sys.path.insert(0, os.path.dirname(HERE))
    from test_pagerank_oracle import out_lists, random_graph

    P = ctypes.c_void_p
    ref = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_pagerank.so"))
    out = {}
    for idx, (n, e, iters) in enumerate([(64, 400, 1), (700, 9000, 3)]):
        src, dst = random_graph(n, e, 7 * n + e)
        out_ptr, out_dst, _ = out_lists(src, dst, n)
        expect = np.zeros(n, np.float32)
        assert ref.ref_pagerank(out_ptr.ctypes.data_as(P), out_dst.ctypes.data_as(P), n, iters,
                                ctypes.c_float(1.0 / n), expect.ctypes.data_as(P)) == 0
        out[f"g{idx}_meta"] = np.array([n, e, iters], np.int64)
        out[f"g{idx}_src"], out[f"g{idx}_dst"], out[f"g{idx}_rank"] = src, dst, expect
    np.savez_compressed(os.path.join(HERE, "pagerank_golden.npz"), **out)


if __name__ == "__main__":
    main()
    main_blas()
    main_scan_sort()
    main_reduce()
    main_pagerank()
