"""GPU parity tests of the imageFilter stencil kernel (through the C ABI).

Every output is compared byte-for-byte with the oracle (itself pinned to the
reference's imageFilter_cpu) on the same seeded inputs: whole images, batched
subtask rectangles, COMPACT (per-subtask copied) views, every filter radius
the reference allows (1..15), both accumulation modes, and the full
8192 x 8192 RGB configuration.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ptr
from test_imgf_oracle import golden_cases, run_oracle

pytestmark = pytest.mark.gpu


def make_case(W, H, R, seed, mode):
    rng = np.random.default_rng(seed)
    img = rng.integers(0, 256, size=H * W * 3, dtype=np.uint8)
    f = np.zeros((32, 32), np.int8)
    lo, hi = (-128, 128) if mode == 0 else (-4, 5)
    f[: 2 * R + 1, : 2 * R + 1] = rng.integers(lo, hi, size=(2 * R + 1, 2 * R + 1))
    return img, f


def gpu_full(torch, img, W, H, R, f, mode, plain=False):
    from unicorn_b200 import ops

    d_in = torch.from_numpy(img).cuda()
    d_out = torch.zeros_like(d_in)
    fn = ops.image_filter_plain if plain else ops.image_filter
    fn(d_in, d_out, W, H, f[: 2 * R + 1, : 2 * R + 1], mode)
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("W,H,R", [(37, 35, 1), (67, 41, 2), (130, 70, 3), (257, 129, 4), (96, 50, 5),
                                   (20, 20, 15), (5, 3, 2), (1, 1, 1), (64, 32, 2), (65, 33, 2)])
def test_full_image_matches_oracle(cuda, oracle, mode, W, H, R):
    img, f = make_case(W, H, R, W * 7 + H + R, mode)
    got = gpu_full(cuda, img, W, H, R, f, mode)
    assert np.array_equal(got, run_oracle(oracle, img, W, H, R, f, mode))


@pytest.mark.parametrize("R", list(range(1, 16)))
def test_every_radius(cuda, oracle, R):
    W, H = 150, 77
    for mode in (0, 1):
        img, f = make_case(W, H, R, 100 + R, mode)
        assert np.array_equal(gpu_full(cuda, img, W, H, R, f, mode),
                              run_oracle(oracle, img, W, H, R, f, mode)), (R, mode)


def test_golden_fixtures_on_gpu(cuda):
    for W, H, R, img, f, expect in golden_cases():
        assert np.array_equal(gpu_full(cuda, img, W, H, R, f, 0), expect), (W, H, R)


@pytest.mark.parametrize("mode", [0, 1])
def test_plain_form_matches_oracle(cuda, oracle, mode):
    W, H, R = 300, 211, 2
    img, f = make_case(W, H, R, 5, mode)
    assert np.array_equal(gpu_full(cuda, img, W, H, R, f, mode, plain=True),
                          run_oracle(oracle, img, W, H, R, f, mode))


def tiles(W, H, T):
    return [(r, min(r + T, H), c, min(c + T, W)) for r in range(0, H, T) for c in range(0, W, T)]


@pytest.mark.parametrize("T", [512, 100, 33])
def test_batched_subtask_rectangles(cuda, oracle, T):
    from unicorn_b200 import ops

    W, H, R = 1030, 777, 2
    img, f = make_case(W, H, R, T, 0)
    rects = tiles(W, H, T)[:256]
    d_in = cuda.from_numpy(img).cuda()
    d_out = cuda.zeros_like(d_in)
    ops.image_filter(d_in, d_out, W, H, f[:5, :5], 0, items=rects)
    cuda.cuda.synchronize()
    got = d_out.cpu().numpy().reshape(H, W, 3)
    ref = run_oracle(oracle, img, W, H, R, f, 0).reshape(H, W, 3)
    covered = np.zeros((H, W), bool)
    for (r0, r1, c0, c1) in rects:
        covered[r0:r1, c0:c1] = True
        assert np.array_equal(got[r0:r1, c0:c1], ref[r0:r1, c0:c1]), (r0, c0)
    assert (got[~covered] == 0).all(), "kernel wrote outside its rectangles"


@pytest.mark.parametrize("R", [2, 3])
@pytest.mark.parametrize("T", [96, 64, 45])
def test_checkerboard_items_two_outputs(cuda, oracle, pmb, T, R):
    """Neighbouring subtasks write to two different output images, so no two
    items of the launch merge: the kernel walks many tensor-map items (item
    changes inside a CTA's tile range, partial tiles at every seam), in the
    interleaved-byte form (R = 2) and the planar form (R = 3)."""
    from unicorn_b200 import capi

    W, H = 1024, 700
    img, f = make_case(W, H, R, 500 + T + R, 1)
    ref = run_oracle(oracle, img, W, H, R, f, 1).reshape(H, W, 3)
    d_in = cuda.from_numpy(img).cuda()
    outs = [cuda.zeros_like(d_in), cuda.zeros_like(d_in)]
    rects = tiles(W, H, T)[:256]
    items = (capi.ImgfItem * len(rects))()
    for k, (r0, r1, c0, c1) in enumerate(rects):
        it = items[k]
        it.in_ = d_in.data_ptr()
        it.out = outs[((r0 // T) + (c0 // T)) & 1].data_ptr()
        it.in_pitch = it.out_pitch = 3 * W
        it.width, it.height = W, H
        it.in_row0 = it.in_col0 = it.out_row0 = it.out_col0 = 0
        it.r0, it.r1, it.c0, it.c1 = r0, r1, c0, c1
    cover = (capi.ImgfItem * len(rects))()
    n = ctypes.c_int(0)
    assert pmb.pmb_image_filter_cover(items, len(rects), cover, ctypes.byref(n)) == 0
    assert n.value == len(rects)
    capi.check(pmb.pmb_image_filter(items, len(rects), ptr(f), R, 1, None))
    cuda.cuda.synchronize()
    got = [o.cpu().numpy().reshape(H, W, 3) for o in outs]
    written = [np.zeros((H, W), bool), np.zeros((H, W), bool)]
    for (r0, r1, c0, c1) in rects:
        o = ((r0 // T) + (c0 // T)) & 1
        written[o][r0:r1, c0:c1] = True
        assert np.array_equal(got[o][r0:r1, c0:c1], ref[r0:r1, c0:c1]), (r0, c0)
    for o in range(2):
        assert (got[o][~written[o]] == 0).all(), "kernel wrote outside its rectangles"


@pytest.mark.parametrize("R", [1, 2, 7])
def test_compact_views(cuda, oracle, pmb, R):
    """Each subtask reads a compact copy of its input subscription and writes a
    compact output block, as the stub stages them for COMPACT visibility."""
    from unicorn_b200 import capi

    W, H, T = 301, 203, 64
    img, f = make_case(W, H, R, 77 + R, 1)
    ref = run_oracle(oracle, img, W, H, R, f, 1).reshape(H, W, 3)
    full = img.reshape(H, W * 3)
    rects = tiles(W, H, T)
    items = (capi.ImgfItem * len(rects))()
    keep = []
    for k, (r0, r1, c0, c1) in enumerate(rects):
        fr, lr = max(0, r0 - R), min(H - 1, r1 - 1 + R)
        fc, lc = max(0, c0 - R), min(W - 1, c1 - 1 + R)
        sub = np.ascontiguousarray(full[H - 1 - lr:H - fr, 3 * fc:3 * (lc + 1)])
        d_sub = cuda.from_numpy(sub.reshape(-1)).cuda()
        d_o = cuda.zeros((r1 - r0) * (c1 - c0) * 3, dtype=cuda.uint8, device="cuda")
        keep.append((d_sub, d_o))
        it = items[k]
        it.in_, it.out = d_sub.data_ptr(), d_o.data_ptr()
        it.in_pitch, it.out_pitch = 3 * (lc - fc + 1), 3 * (c1 - c0)
        it.width, it.height = W, H
        it.in_row0, it.in_col0 = H - 1 - lr, fc
        it.out_row0, it.out_col0 = r0, c0
        it.r0, it.r1, it.c0, it.c1 = r0, r1, c0, c1
    capi.check(pmb.pmb_image_filter(items, len(rects), ptr(f), R, 1, None))
    cuda.cuda.synchronize()
    for (r0, r1, c0, c1), (_, d_o) in zip(rects, keep):
        got = d_o.cpu().numpy().reshape(r1 - r0, c1 - c0, 3)
        assert np.array_equal(got, ref[r0:r1, c0:c1]), (r0, c0)


@pytest.mark.parametrize("mode", [1, 0])
def test_full_configuration_8192(cuda, oracle, mode):
    """8192 x 8192 RGB, 5x5 filter, 512 x 512 subtasks in one launch."""
    from unicorn_b200 import ops

    W = H = 8192
    R = 2
    img, f = make_case(W, H, R, 3, mode)
    d_in = cuda.from_numpy(img).cuda()
    d_out = cuda.zeros_like(d_in)
    ops.image_filter(d_in, d_out, W, H, f[:5, :5], mode, items=tiles(W, H, 512))
    cuda.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy(), run_oracle(oracle, img, W, H, R, f, mode))


def test_zz_stencil_error_word_clear(cuda, pmb):
    """Last in this file: no bounded wait of any tensor-core stencil launch
    above expired (the error word is sticky until cleared)."""
    err = ctypes.c_uint32(0xFFFFFFFF)
    assert pmb.pmb_image_filter_error(1, ctypes.byref(err)) == 0
    assert err.value == 0
