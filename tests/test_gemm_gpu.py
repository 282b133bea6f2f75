"""GPU tests of the tcgen05 BF16x3 GEMM and the plain FP32 SIMT GEMM.

The FP64 oracle is numpy float64 matmul of the same fp32 inputs.  Bars:
normwise ||C - C64||_F / ||C64||_F <= 1e-5 (the configuration's accuracy
target) and elementwise |dC_ij| <= 2^-15 (|A||B|)_ij; the workspace error word
must stay 0.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NORM_TOL = 1e-5
ELEM_TOL = 2.0 ** -15


def mats(M, N, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    return A, B


def errors(got, A, B, C0=None, alpha=1.0, beta=0.0):
    ref = alpha * (A.astype(np.float64) @ B.astype(np.float64))
    if C0 is not None and beta != 0.0:
        ref += beta * C0.astype(np.float64)
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    norm = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300)
    elem = np.max(np.abs(got - ref) / np.maximum(abs(alpha) * scale, 1e-30))
    return norm, elem


def run(cuda, A, B, C0=None, alpha=1.0, beta=0.0, plain=False):
    from unicorn_b200 import ops

    dA, dB = cuda.from_numpy(A).cuda(), cuda.from_numpy(B).cuda()
    dC = cuda.from_numpy(C0).cuda() if C0 is not None else None
    C, ws = ops.sgemm(dA, dB, dC, alpha, beta, plain=plain)
    cuda.cuda.synchronize()
    if ws is not None:
        assert ops.scratch_error(ws) == 0
    return C.cpu().numpy()


@pytest.mark.parametrize("M,N,K", [(128, 256, 32), (256, 256, 1024), (1, 1, 1), (100, 300, 77), (129, 257, 33),
                                   (300, 520, 640), (1024, 1024, 1024)])
def test_bf16x3_matches_fp64(cuda, M, N, K):
    A, B = mats(M, N, K, M + N + K)
    norm, elem = errors(run(cuda, A, B), A, B)
    assert norm <= NORM_TOL and elem <= ELEM_TOL, (norm, elem)


def test_bf16x3_long_k(cuda):
    A, B = mats(256, 512, 8192, 5)
    norm, elem = errors(run(cuda, A, B), A, B)
    assert norm <= NORM_TOL and elem <= ELEM_TOL, (norm, elem)


@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (0.5, -2.0), (2.0, 0.0)])
def test_alpha_beta_epilogue(cuda, alpha, beta):
    M, N, K = 384, 512, 256
    A, B = mats(M, N, K, 9)
    C0 = np.random.default_rng(1).uniform(-1, 1, (M, N)).astype(np.float32)
    norm, elem = errors(run(cuda, A, B, C0, alpha, beta), A, B, C0, alpha, beta)
    assert norm <= NORM_TOL, norm


def test_submatrix_views_with_leading_dimensions(cuda):
    """A row block of A and a column block of B inside larger matrices (the
    NATURAL view of a matrixMultiply subtask: lda = ldb = ldc = n)."""
    from unicorn_b200 import ops

    n, blk = 1024, 256
    A, B = mats(n, n, n, 3)
    dA, dB = cuda.from_numpy(A).cuda(), cuda.from_numpy(B).cuda()
    dC = cuda.zeros(n, n, device="cuda")
    for row in range(n // blk):
        for col in range(n // blk):
            ops.sgemm(dA[row * blk:(row + 1) * blk], dB[:, col * blk:(col + 1) * blk],
                      dC[row * blk:(row + 1) * blk, col * blk:(col + 1) * blk])
    cuda.cuda.synchronize()
    norm, elem = errors(dC.cpu().numpy(), A, B)
    assert norm <= NORM_TOL and elem <= ELEM_TOL, (norm, elem)


@pytest.mark.parametrize("M,N,K,alpha,beta", [(300, 520, 64, -1.0, 1.0), (1000, 1536, 40, 0.5, -2.0),
                                              (256, 256, 16, 1.0, 0.0), (77, 1000, 64, -1.0, 1.0),
                                              (2000, 4, 8, 2.0, 1.0)])
def test_short_k_update(cuda, M, N, K, alpha, beta):
    """K <= 64 with an aligned C takes the kernel that moves C by TMA (the LU
    trailing update's shape); ragged M and N exercise its clipped boxes."""
    A, B = mats(M, N, K, 11 + M)
    C0 = np.random.default_rng(M + N).uniform(-1, 1, (M, N)).astype(np.float32)
    norm, elem = errors(run(cuda, A, B, C0, alpha, beta), A, B, C0, alpha, beta)
    assert norm <= NORM_TOL, norm


def test_short_k_update_into_view_leaves_the_rest(cuda):
    """C as an aligned view inside a larger matrix: only the view changes."""
    from unicorn_b200 import ops

    M, N, K = 300, 520, 64
    A, B = mats(M, N, K, 21)
    big = np.random.default_rng(5).uniform(-1, 1, (600, 800)).astype(np.float32)
    dbig = cuda.from_numpy(big.copy()).cuda()
    view = dbig[8:8 + M, 16:16 + N]
    _, ws = ops.sgemm(cuda.from_numpy(A).cuda(), cuda.from_numpy(B).cuda(), view, -1.0, 1.0)
    cuda.cuda.synchronize()
    assert ops.scratch_error(ws) == 0
    got = dbig.cpu().numpy()
    norm, _ = errors(got[8:8 + M, 16:16 + N], A, B, big[8:8 + M, 16:16 + N], -1.0, 1.0)
    assert norm <= NORM_TOL, norm
    mask = np.ones_like(big, dtype=bool)
    mask[8:8 + M, 16:16 + N] = False
    assert np.array_equal(got[mask], big[mask])


@pytest.mark.parametrize("M,N,K", [(64, 64, 64), (100, 300, 77), (512, 512, 512)])
def test_plain_sgemm(cuda, M, N, K):
    A, B = mats(M, N, K, 2)
    norm, _ = errors(run(cuda, A, B, plain=True), A, B)
    assert norm <= NORM_TOL, norm


def test_k_zero_scales_c(cuda):
    from unicorn_b200 import ops

    C0 = np.ones((4, 5), np.float32)
    dA = cuda.zeros(4, 0, device="cuda")
    dB = cuda.zeros(0, 5, device="cuda")
    dC = cuda.from_numpy(C0).cuda()
    ops.sgemm(dA, dB, dC, 1.0, 3.0)
    cuda.cuda.synchronize()
    assert np.allclose(dC.cpu().numpy(), 3.0)


@pytest.mark.parametrize("M,N,K", [(1024, 1024, 1024), (300, 520, 64)])
def test_product_after_producer_on_same_stream(cuda, M, N, K):
    """The product kernel is a programmatic dependent of the split pass; the
    split pass itself must wait for a kernel that writes A earlier on the
    stream."""
    from unicorn_b200 import ops

    A, B = mats(M, N, K, 41)
    srcA = cuda.from_numpy(A).cuda()
    dA = cuda.zeros_like(srcA)
    dB = cuda.from_numpy(B).cuda()
    s = cuda.cuda.Stream()
    with cuda.cuda.stream(s):
        dA.copy_(srcA)
        C, ws = ops.sgemm(dA, dB, stream=s)
        dA.zero_()
    s.synchronize()
    norm, _ = errors(C.cpu().numpy(), A, B)
    assert norm <= NORM_TOL, norm


AUTOTUNE_SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from unicorn_b200 import ops
rng = np.random.default_rng(1)
worst = 0.0
for (M, N, K) in [(1024, 1024, 1024), (1024, 1024, 1024), (300, 2000, 700), (4096, 512, 256), (96, 96, 4096)]:
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    C, ws = ops.sgemm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda())
    torch.cuda.synchronize()
    assert ops.scratch_error(ws) == 0
    ref = A.astype(np.float64) @ B.astype(np.float64)
    worst = max(worst, float(np.linalg.norm(C.cpu().numpy() - ref) / np.linalg.norm(ref)))
print("worst", worst)
"""


def test_autotuned_products_match_fp64():
    """PMB_GEMM_AUTOTUNE=1: the first product of a shape class times the three
    product kernels on its own operands (C written by each in turn) and keeps
    the fastest; every result, tuned or cached, meets the normwise bar."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", AUTOTUNE_SCRIPT, root], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, PMB_GEMM_AUTOTUNE="1"))
    assert p.returncode == 0, p.stdout + p.stderr
    worst = float(p.stdout.split("worst")[-1])
    assert worst <= NORM_TOL, worst
