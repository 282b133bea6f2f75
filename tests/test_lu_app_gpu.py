"""luDecomposition on the GPU through the reference app's own stage tasks.

* pmb_trsm_f32 (the HORZ_VERT_COMP solves) against FP64 numpy solves, both
  forms the app uses (left/lower/non-unit, right/upper/unit) and the other
  diagonal kind, on ragged sizes.
* The reference app's DoParallelProcess (luDecomposition.cpp:425-470,
  compiled unchanged, oracle/_ref/libref_lu_gpu.so) run through the B200
  runtime with the B200 GPU callbacks (libpmb_app_luDecomposition.so): its
  factors must match the FP64 Crout oracle (restating serialLUDecomposition)
  elementwise and by FP64 residual ||A - LU||_F / ||A||_F <= 1e-5.
* The unchanged app binary in parallel mode 2 (its stage tasks on the GPU
  stub) completes; it does not compare fp32 results itself
  (luDecomposition.cpp:593-595).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, ptr
from test_lu import crout_f64, dd_matrix

pytestmark = pytest.mark.gpu

LU_GLUE = os.path.join(ROOT, "oracle", "_ref", "libref_lu_gpu.so")
LU_APP = os.path.join(ROOT, "oracle", "_ref", "luDecomposition_b200.exe")


@pytest.mark.parametrize("side,unit,m,n", [("left", False, 300, 77), ("left", True, 129, 64),
                                           ("left", False, 2048, 2048), ("right", True, 300, 77),
                                           ("right", False, 65, 200), ("right", True, 2048, 2048)])
def test_trsm_matches_fp64(cuda, pmb, side, unit, m, n):
    from unicorn_b200 import capi, ops

    rng = np.random.default_rng(m * 7 + n)
    order = m if side == "left" else n
    # Off-diagonal entries of size 1/order, as in the factors of a diagonally
    # dominant matrix: a unit triangle of O(1) random entries has an inverse
    # that grows like 2^order.
    T = (rng.uniform(-1, 1, (order, order)) / order).astype(np.float32)
    T[np.arange(order), np.arange(order)] += 1.0
    B = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    # column-major device copies: element (r, c) at [c, r]
    dA = cuda.from_numpy(np.ascontiguousarray(T.T)).cuda()
    dB = cuda.from_numpy(np.ascontiguousarray(B.T)).cuda()
    s = capi.PMB_SIDE_LEFT if side == "left" else capi.PMB_SIDE_RIGHT
    uplo = capi.PMB_FILL_LOWER if side == "left" else capi.PMB_FILL_UPPER
    diag = capi.PMB_DIAG_UNIT if unit else capi.PMB_DIAG_NON_UNIT
    wsb = pmb.pmb_trsm_workspace_bytes(s, m, n)
    ws = ops._scratch(wsb)
    capi.check(pmb.pmb_trsm_f32(s, uplo, diag, m, n, dA.data_ptr(), order, dB.data_ptr(), m, ws.data_ptr(), wsb,
                                cuda.cuda.current_stream().cuda_stream))
    cuda.cuda.synchronize()
    X = dB.cpu().numpy().T.astype(np.float64)
    T64 = T.astype(np.float64)
    if side == "left":
        L = np.tril(T64)
        if unit:
            np.fill_diagonal(L, 1.0)
        ref = np.linalg.solve(L, B.astype(np.float64))
    else:
        U = np.triu(T64)
        if unit:
            np.fill_diagonal(U, 1.0)
        ref = np.linalg.solve(U.T, B.astype(np.float64).T).T
    err = np.linalg.norm(X - ref) / np.linalg.norm(ref)
    assert err <= 1e-5, err


def test_trsm_rejects_unprovided_forms(pmb):
    from unicorn_b200 import capi

    st = pmb.pmb_trsm_f32(capi.PMB_SIDE_LEFT, capi.PMB_FILL_UPPER, capi.PMB_DIAG_UNIT, 4, 4, ctypes.c_void_p(256), 4,
                          ctypes.c_void_p(256), 4, ctypes.c_void_p(256), 1 << 20, None)
    assert st == capi.PMB_INVALID_INDEX


@pytest.mark.parametrize("n", [4096, 6144])
def test_reference_lu_app_stages_on_gpu(cuda, oracle, n):
    if not os.path.exists(LU_GLUE):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    glue = ctypes.CDLL(LU_GLUE)
    a = dd_matrix(n, 70 + n)  # column-major: row index of the array = column of the matrix
    got = a.copy()
    assert glue.ref_lu_app_gpu(ptr(got), ctypes.c_ulong(n)) == 0
    if n == 4096:  # the FP64 Crout oracle is one thread (about 25 s here); larger n checks the residual
        ref = crout_f64(oracle, a)
        assert np.allclose(got, ref, rtol=1e-4, atol=1e-5)
    from unicorn_b200 import ops

    d0 = cuda.from_numpy(a).cuda()
    dlu = cuda.from_numpy(got).cuda()
    assert ops.lu_residual(d0, dlu) <= 1e-5


def test_reference_lu_app_binary_gpu_mode():
    if not os.path.exists(LU_APP):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    p = subprocess.run([LU_APP, "1", "2", "0", "4096"], capture_output=True, text=True, timeout=600)
    out = p.stdout + p.stderr
    assert p.returncode == 0 and "Parallel Task 2 Execution Time" in out and "Failed" not in out, out
