"""LU tests.  CPU: the FP64 Crout oracle (restating serialLUDecomposition)
reconstructs A.  GPU: the blocked tensor-core LU and the plain FP32 form
against that oracle (elementwise) and by FP64 residual ||A - LU||/||A||."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ptr


def dd_matrix(n, seed):
    """Diagonally dominant test matrix: U[-1,1] plus n on the diagonal."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    a[np.arange(n), np.arange(n)] += n
    return a  # interpreted column-major: element (r, c) at a.T[r, c]


def crout_f64(oracle, a_cm):
    """a_cm: (n, n) array holding the column-major matrix (row index = column)."""
    n = a_cm.shape[0]
    x = np.ascontiguousarray(a_cm, dtype=np.float64)
    oracle.orc_lu_crout_f64(ptr(x), n, ctypes.c_long(n))
    return x


def reconstruct(lu_cm):
    lu = lu_cm.T.astype(np.float64)  # (row, col)
    L = np.tril(lu)
    U = np.triu(lu, 1) + np.eye(lu.shape[0])
    return L @ U


@pytest.mark.parametrize("n", [1, 2, 7, 64, 150])
def test_oracle_reconstructs(oracle, n):
    a = dd_matrix(n, n)
    lu = crout_f64(oracle, a)
    A = a.T.astype(np.float64)
    assert np.linalg.norm(reconstruct(lu) - A) / np.linalg.norm(A) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("n,nb", [(1, 128), (5, 4), (64, 32), (100, 64), (128, 128), (129, 128), (300, 64),
                                  (512, 128), (1000, 96), (1001, 64), (515, 48), (257, 64)])
def test_gpu_lu_matches_oracle(cuda, oracle, n, nb):
    from unicorn_b200 import ops

    a = dd_matrix(n, 10 + n)
    d = cuda.from_numpy(a.copy()).cuda()
    d0 = cuda.from_numpy(a.copy()).cuda()
    _, ws, flags = ops.lu_decompose(d, nb)
    assert flags == 0
    got = d.cpu().numpy()
    ref = crout_f64(oracle, a)
    assert np.allclose(got, ref, rtol=1e-4, atol=1e-5)
    assert ops.lu_residual(d0, d) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("nb", [128, 64])
def test_gpu_lu_plain_form(cuda, oracle, nb):
    from unicorn_b200 import ops

    n = 700
    a = dd_matrix(n, 4)
    d = cuda.from_numpy(a.copy()).cuda()
    d0 = cuda.from_numpy(a.copy()).cuda()
    ops.lu_decompose(d, nb, plain=True)
    assert ops.lu_residual(d0, d) <= 1e-5
    assert np.allclose(d.cpu().numpy(), crout_f64(oracle, a), rtol=1e-4, atol=1e-5)


@pytest.mark.gpu
def test_pivot_check_flags_non_dominant_matrix(cuda):
    from unicorn_b200 import ops

    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, (200, 200)).astype(np.float32)
    a[np.arange(200), np.arange(200)] += 3.0  # not dominant enough: partial pivoting would swap
    d = cuda.from_numpy(a).cuda()
    _, _, flags = ops.lu_decompose(d, 64)
    assert flags & 1


@pytest.mark.gpu
@pytest.mark.parametrize("row", [10, 150])
def test_pivot_check_one_large_entry(cuda, row):
    """One L entry larger than its pivot, inside the diagonal block (row 10)
    or below it (row 150): both halves of the check must see it."""
    from unicorn_b200 import ops

    n = 200
    a = dd_matrix(n, 7)
    a[5, row] = 10.0 * n  # memory is column-major: matrix element (row, 5)
    d = cuda.from_numpy(a).cuda()
    _, _, flags = ops.lu_decompose(d, 64)
    assert flags & 1


@pytest.mark.gpu
@pytest.mark.parametrize("n,nb", [(2048, 128), (4096, 128), (4096, 64)])
def test_gpu_lu_large_residual(cuda, n, nb):
    from unicorn_b200 import ops

    a = dd_matrix(n, n)
    d = cuda.from_numpy(a.copy()).cuda()
    d0 = cuda.from_numpy(a).cuda()
    _, _, flags = ops.lu_decompose(d, nb)
    assert flags == 0
    assert ops.lu_residual(d0, d) <= 1e-5


@pytest.mark.gpu
def test_gpu_lu_after_producer_on_same_stream(cuda, oracle):
    """The block steps are chained by programmatic dependent launch; the first
    step must still wait for a kernel that writes A earlier on the same stream
    (no host synchronisation in between), and a second factorization queued
    right behind the first must see its own input."""
    from unicorn_b200 import ops

    n = 1000
    a = dd_matrix(n, 31)
    src = cuda.from_numpy(a.copy()).cuda()
    d = cuda.zeros_like(src)
    s = cuda.cuda.Stream()
    with cuda.cuda.stream(s):
        d.copy_(src)                     # the producer, on s
        _, ws, _ = ops.lu_decompose(d, 64, stream=s)
        d2 = d.clone()                   # reads the first result on s
        d.copy_(src)                     # a fresh input, on s again
        ops.lu_decompose(d, 64, workspace=ws, stream=s)
    s.synchronize()
    ref = crout_f64(oracle, a)
    assert np.allclose(d.cpu().numpy(), ref, rtol=1e-4, atol=1e-5)
    assert np.allclose(d2.cpu().numpy(), ref, rtol=1e-4, atol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [100, 1000, 2048])
def test_fp64_refinement_recovers_fp64_accuracy(cuda, pmb, n):
    """Refined solves with the BF16x3/FP64 LU factors: the backward error
    falls from fp32 level to FP64 level, and x matches an FP64 solve."""
    from unicorn_b200 import capi, ops

    a = dd_matrix(n, 500 + n)
    d0 = cuda.from_numpy(a.copy()).cuda()
    d = cuda.from_numpy(a.copy()).cuda()
    ops.lu_decompose(d, 64)
    b = np.random.default_rng(n).uniform(-1, 1, n)
    db = cuda.from_numpy(b).cuda()
    dx = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    iters = 4
    berr = cuda.zeros(iters + 1, dtype=cuda.float64, device="cuda")
    wsb = pmb.pmb_lu_refine_workspace_bytes(n)
    ws = ops._scratch(wsb)
    capi.check(pmb.pmb_lu_solve_refined(d0.data_ptr(), n, d.data_ptr(), n, n, db.data_ptr(), dx.data_ptr(), iters,
                                        berr.data_ptr(), ws.data_ptr(), wsb, cuda.cuda.current_stream().cuda_stream))
    cuda.cuda.synchronize()
    e = berr.cpu().numpy()
    assert e[0] < 1e-5 and e[-1] < 1e-14, e
    A = a.T.astype(np.float64)
    ref = np.linalg.solve(A, b)
    x = dx.cpu().numpy()
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-12
