"""GEMM and LU oracles pinned to the reference's own CPU callbacks.

The reference computes matrixMultiplyBlas and luDecomposition in a CBLAS that
is not part of its tree; its CPU callbacks (matrixMultiplyBlas.cpp,
luDecomposition.cpp) are compiled unchanged into oracle/_ref/libref_mm.so and
libref_lu.so over a CBLAS shim on numpy's OpenBLAS (oracle/ref/Makefile).

* With the reference tree built here: the reference's task of (n/block)^2 GEMM
  subtasks and its three-stage blocked LU (LU_DECOMPOSE / HORZ_VERT_COMP /
  DIAGONAL_COMP, BLOCK_DIM 2048) are checked against the FP64 oracles with the
  same bars the B200 kernels are held to (GEMM: normwise 1e-5 and 2^-15
  (|A||B|) elementwise; LU: rtol 1e-4 / atol 1e-5 against the FP64 Crout
  factors, FP64 residual <= 1e-5); serialLUDecomposition equals the restated
  orc_lu_crout_f64 within fp32 rounding.
* Everywhere: the golden vectors tests/golden/blas_golden.npz (written from
  those libraries by tests/golden/make_golden.py) against the oracles, and the
  GEMM subscription geometry of matrixMultiplyDataDistribution against its
  restatement.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT, ptr

GOLDEN = os.path.join(ROOT, "tests", "golden", "blas_golden.npz")


def _lib(name):
    path = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    return ctypes.CDLL(path)


@pytest.fixture(scope="module")
def ref_mm():
    return _lib("libref_mm.so")


@pytest.fixture(scope="module")
def ref_lu():
    return _lib("libref_lu.so")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def gemm_bars(a, b, c):
    """The GEMM parity bars of the B200 kernel tests, against FP64."""
    a64, b64 = a.astype(np.float64), b.astype(np.float64)
    c64 = a64 @ b64
    rel = np.linalg.norm(c.astype(np.float64) - c64) / np.linalg.norm(c64)
    elem = np.abs(c.astype(np.float64) - c64) <= 2.0 ** -15 * (np.abs(a64) @ np.abs(b64)) + 1e-30
    return rel, bool(elem.all())


def dd_cols(n, ld, seed):
    """Column-major n x n diagonally dominant matrix with column stride ld:
    row k of the (n, ld) array is column k; U[-1,1] plus n on the diagonal."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (n, ld)).astype(np.float32)
    a[np.arange(n), np.arange(n)] += n
    return a


def crout_f64(oracle, a_cols, n, ld):
    x = np.ascontiguousarray(a_cols, dtype=np.float64)
    oracle.orc_lu_crout_f64(ptr(x), n, ctypes.c_long(ld))
    return x


def restated_mm_subscriptions(n, block, sid):
    """matrixMultiplyDataDistribution (matrixMultiplyBlas.cpp:90-113), unsplit:
    subtask ids run down the block columns of C (row = id % nb, col = id / nb);
    A: the block row, B: the block column, C: the block.  Rows of
    {type, offset, size, step, count} per memory index (READ = 0, WRITE = 1)."""
    nb = n // block
    row, col = sid % nb, sid // nb
    return [0, row * block * n * 4, n * 4, n * 4, block,
            0, col * block * 4, block * 4, n * 4, n,
            1, (row * n + col) * block * 4, block * 4, n * 4, block]


# ---------------------------------------------------------------- golden


def test_golden_gemm_matches_fp64_oracle(golden):
    k = 0
    while f"mm{k}_meta" in golden.files:
        a, b, c = golden[f"mm{k}_a"], golden[f"mm{k}_b"], golden[f"mm{k}_c"]
        rel, elem_ok = gemm_bars(a, b, c)
        assert rel <= 1e-6 and elem_ok, (k, rel)
        k += 1
    assert k == 2


def test_golden_lu_matches_restated_oracle(oracle, golden):
    k = 0
    while f"lu{k}_meta" in golden.files:
        n, ld, _ = (int(x) for x in golden[f"lu{k}_meta"])
        a, ref = golden[f"lu{k}_in"], golden[f"lu{k}_out"]
        got = crout_f64(oracle, a, n, ld)
        assert np.allclose(ref[:, :n], got[:, :n], rtol=1e-4, atol=1e-5), k
        assert np.array_equal(ref[:, n:], a[:, n:]), "bytes past the leading block changed"
        k += 1
    assert k == 2


def test_golden_gemm_subscriptions(golden):
    for idx in range(2):
        n, block = (int(x) for x in golden[f"mmsub{idx}_meta"])
        rows = golden[f"mmsub{idx}"]
        assert rows.shape[0] == (n // block) ** 2
        for sid in range(rows.shape[0]):
            assert [int(x) for x in rows[sid]] == restated_mm_subscriptions(n, block, sid), (n, block, sid)


# ---------------------------------------------------------------- reference tree


def test_reference_block_sizes(ref_mm, ref_lu):
    assert ref_mm.ref_mm_block_dim() == 2048
    ref_lu.ref_lu_block_dim.restype = ctypes.c_ulong
    assert ref_lu.ref_lu_block_dim() == 2048
    ref_mm.ref_mm_block_size.restype = ctypes.c_ulong
    assert [ref_mm.ref_mm_block_size(ctypes.c_ulong(n)) for n in (256, 1024, 2048, 8192)] == [256, 1024, 2048, 2048]


@pytest.mark.parametrize("n,block,seed", [(1024, 256, 0), (2048, 512, 3), (4096, 2048, 4)])
def test_reference_gemm_task_meets_kernel_bars(ref_mm, n, block, seed):
    """The 1024 task in 256 x 256 subtasks is the CPU-runnable configuration."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    b = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    c = np.full_like(a, np.nan)
    assert ref_mm.ref_mm_task(ptr(a), ptr(b), ptr(c), ctypes.c_ulong(n), ctypes.c_ulong(block)) == 0
    rel, elem_ok = gemm_bars(a, b, c)
    assert rel <= 1e-5 and elem_ok, rel


@pytest.mark.parametrize("n,ld", [(1, 1), (2, 3), (7, 9), (64, 64), (200, 233)])
def test_reference_serial_lu_equals_restated_oracle(oracle, ref_lu, n, ld):
    """serialLUDecomposition (fp32 BLAS) and orc_lu_crout_f64 (FP64 loops):
    same Crout split, L with the diagonal, unit U above it."""
    a = dd_cols(n, ld, 100 + n)
    r = a.copy()
    assert ref_lu.ref_lu_serial(ptr(r), ctypes.c_ulong(n), ctypes.c_ulong(ld)) == 0
    got = crout_f64(oracle, a, n, ld)
    assert np.allclose(r[:, :n], got[:, :n], rtol=1e-4, atol=1e-5)
    assert np.array_equal(r[:, n:], a[:, n:])


def test_reference_blocked_lu_meets_kernel_bars(ref_lu):
    """The reference app's three stages over 2 x 2 blocks of 2048 against the
    FP64 Crout factors (from LAPACK's LU: partial pivoting keeps P = I on a
    diagonally dominant matrix; Doolittle L, U rescaled by diag(U))."""
    scipy_linalg = pytest.importorskip("scipy.linalg")
    n = 4096
    a = dd_cols(n, n, 5)
    r = a.copy()
    assert ref_lu.ref_lu_blocked(ptr(r), ctypes.c_ulong(n)) == 0
    A = a.T.astype(np.float64)  # (row, col)
    lu, piv = scipy_linalg.lu_factor(A)
    assert np.array_equal(piv, np.arange(n))
    d = np.diag(lu).copy()
    crout = np.tril(np.tril(lu, -1) + np.eye(n)) * d[None, :] + np.triu(lu / d[:, None], 1)
    got = r.T.astype(np.float64)
    assert np.allclose(got, crout, rtol=1e-4, atol=1e-5)
    L, U = np.tril(got), np.triu(got, 1) + np.eye(n)
    assert np.linalg.norm(A - L @ U) / np.linalg.norm(A) <= 1e-5
