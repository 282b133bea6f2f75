"""GPU tests of the grouped BF16x3 GEMM (pmb_sgemm_bf16x3_grouped): every
product of a grouped call meets the bars of a single pmb_sgemm_bf16x3 call
(elementwise <= 2^-15 |A||B| against FP64 for every product; normwise <= 1e-5
for K >= 32 -- with K of a few terms the dropped lo*lo term, up to 2^-16
relative per product, is not averaged out), and equals that single call bit
for bit where both run the 2-SM kernel (the tiles run the same kernel body on
the same split operands)."""
from __future__ import annotations

import numpy as np
import pytest

from test_gemm_gpu import ELEM_TOL, NORM_TOL, errors, mats

pytestmark = pytest.mark.gpu


def grouped(cuda, shapes, alpha=1.0, beta=0.0, seed=0):
    from unicorn_b200 import ops

    host, prods = [], []
    for i, (M, N, K) in enumerate(shapes):
        A, B = mats(M, N, K, seed + 7 * i)
        C0 = np.random.default_rng(seed + i).uniform(-1, 1, (M, N)).astype(np.float32)
        dA, dB, dC = (cuda.from_numpy(x).cuda() for x in (A, B, C0))
        host.append((A, B, C0))
        prods.append((dA, dB, dC, alpha, beta))
    ws = ops.sgemm_grouped(prods)
    cuda.cuda.synchronize()
    assert ops.scratch_error(ws) == 0
    return host, prods


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (0.5, -1.25)])
def test_grouped_mixed_shapes_match_fp64(cuda, alpha, beta):
    shapes = [(256, 256, 1024), (100, 300, 77), (1, 1, 1), (129, 257, 33), (512, 128, 256), (300, 520, 640),
              (1024, 1024, 256), (64, 2048, 96)]
    host, prods = grouped(cuda, shapes, alpha, beta)
    for (A, B, C0), (_, _, dC, _, _) in zip(host, prods):
        norm, elem = errors(dC.cpu().numpy(), A, B, C0, alpha, beta)
        assert elem <= ELEM_TOL and (A.shape[1] < 32 or norm <= NORM_TOL), (A.shape, B.shape, norm, elem)


def test_grouped_more_products_than_one_launch(cuda):
    # 30 products: two product launches (24 per launch), 256-row tiles of both widths.
    rng = np.random.default_rng(3)
    shapes = [(int(rng.integers(1, 600)), int(rng.integers(1, 600)), int(rng.integers(1, 700))) for _ in range(30)]
    host, prods = grouped(cuda, shapes, 1.0, 0.0, seed=11)
    for (A, B, C0), (_, _, dC, _, _) in zip(host, prods):
        norm, elem = errors(dC.cpu().numpy(), A, B)
        assert elem <= ELEM_TOL and (A.shape[1] < 32 or norm <= NORM_TOL), (A.shape, B.shape, norm, elem)


def test_grouped_equals_single_calls(cuda):
    from unicorn_b200 import ops

    shapes = [(512, 512, 512), (256, 768, 1024), (384, 256, 96)]
    host, prods = grouped(cuda, shapes, 1.0, 0.0, seed=5)
    for (A, B, C0), (dA, dB, dC, _, _) in zip(host, prods):
        single, _ = ops.sgemm(dA, dB)
        cuda.cuda.synchronize()
        assert np.array_equal(single.cpu().numpy(), dC.cpu().numpy())


def test_grouped_views_and_k_zero(cuda):
    from unicorn_b200 import ops

    # Products into disjoint blocks of one C (leading dimension 1024), and a K = 0 product (C *= beta).
    big = cuda.zeros(512, 1024, dtype=cuda.float32, device="cuda")
    A, B = mats(512, 512, 300, 9)
    dA, dB = cuda.from_numpy(A).cuda(), cuda.from_numpy(B).cuda()
    left, right = big[:, :512], big[:, 512:]
    z = cuda.ones(64, 64, dtype=cuda.float32, device="cuda")
    empty_a = cuda.zeros(64, 0, dtype=cuda.float32, device="cuda")
    empty_b = cuda.zeros(0, 64, dtype=cuda.float32, device="cuda")
    ws = ops.sgemm_grouped([(dA, dB, left, 1.0, 0.0), (dA, dB, right, 2.0, 0.0), (empty_a, empty_b, z, 1.0, 3.0)])
    cuda.cuda.synchronize()
    assert ops.scratch_error(ws) == 0
    got = big.cpu().numpy()
    for half, alpha in ((got[:, :512], 1.0), (got[:, 512:], 2.0)):
        norm, elem = errors(half, A, B, alpha=alpha)
        assert norm <= NORM_TOL and elem <= ELEM_TOL
    assert np.all(z.cpu().numpy() == 3.0)
