"""CPU tests of pmb_image_filter_cover: the host step that lets one stencil
launch cover a batch of subtasks as the larger rectangles they tile.

Merging must leave the filtered bytes unchanged, so the tests check (a) the
subtask grid of a NATURAL-view task collapses to the image, whatever view
origin each subtask's pointer has, (b) nothing merges across different
images, pitches (COMPACT views) or non-adjacent rectangles, and (c) on random
partitions the merged rectangles cover exactly the same output pixels, each
once, and read and write through the same per-pixel addresses."""
from __future__ import annotations

import ctypes

import numpy as np

from unicorn_b200 import capi

IN_BASE = 0x7F0000000000
OUT_BASE = 0x7E0000000000


def natural_item(W, H, R, r0, r1, c0, c1, in_base=IN_BASE, out_base=OUT_BASE, runtime_origin=True):
    """An item as the imageFiltering callback builds it for a NATURAL view:
    the input pointer at the first buffer row / column of the subscription
    and the output pointer at the rectangle, or both at the image origin."""
    it = capi.ImgfItem()
    pitch = 3 * W
    if runtime_origin:
        last_row = min(H - 1, r1 - 1 + R)
        first_col = max(0, c0 - R)
        it.in_row0, it.in_col0 = H - 1 - last_row, first_col
        it.out_row0, it.out_col0 = r0, c0
    else:
        it.in_row0 = it.in_col0 = it.out_row0 = it.out_col0 = 0
    it.in_ = in_base + it.in_row0 * pitch + 3 * it.in_col0
    it.out = out_base + it.out_row0 * pitch + 3 * it.out_col0
    it.in_pitch = it.out_pitch = pitch
    it.width, it.height = W, H
    it.r0, it.r1, it.c0, it.c1 = r0, r1, c0, c1
    return it


def cover(pmb, items):
    arr = (capi.ImgfItem * len(items))(*items)
    out = (capi.ImgfItem * len(items))()
    n = ctypes.c_int(-1)
    assert pmb.pmb_image_filter_cover(arr, len(items), out, ctypes.byref(n)) == 0, pmb.pmb_last_error()
    assert 0 <= n.value <= len(items)
    return [out[i] for i in range(n.value)]


def rects(items):
    return sorted((it.r0, it.r1, it.c0, it.c1) for it in items)


def in_addr(it, m, n):
    return it.in_ + (it.height - 1 - m - it.in_row0) * it.in_pitch + 3 * (n - it.in_col0)


def out_addr(it, m, n):
    return it.out + (m - it.out_row0) * it.out_pitch + 3 * (n - it.out_col0)


def test_subtask_grid_collapses_to_the_image(pmb):
    W = H = 8192
    items = [natural_item(W, H, 2, r, r + 512, c, c + 512) for r in range(0, H, 512) for c in range(0, W, 512)]
    got = cover(pmb, items)
    assert rects(got) == [(0, H, 0, W)]
    # Every pixel's input and output addresses are those of the subtask that owns it.
    rng = np.random.default_rng(0)
    for _ in range(200):
        m, n = int(rng.integers(0, H)), int(rng.integers(0, W))
        own = items[(m // 512) * 16 + n // 512]
        assert in_addr(got[0], m, n) == in_addr(own, m, n)
        assert out_addr(got[0], m, n) == out_addr(own, m, n)


def test_image_origin_pointers_merge_too(pmb):
    W, H = 1000, 600
    items = [natural_item(W, H, 3, r, r + 200, c, min(c + 256, W), runtime_origin=False)
             for r in range(0, H, 200) for c in range(0, W, 256)]
    assert rects(cover(pmb, items)) == [(0, H, 0, W)]


def test_no_merge_across_images_pitches_or_gaps(pmb):
    W = H = 1024
    a = natural_item(W, H, 2, 0, 512, 0, 512)
    b_other_out = natural_item(W, H, 2, 0, 512, 512, 1024, out_base=OUT_BASE + 0x100000000)
    b_other_in = natural_item(W, H, 2, 0, 512, 512, 1024, in_base=IN_BASE + 0x100000000)
    assert len(cover(pmb, [a, b_other_out])) == 2
    assert len(cover(pmb, [a, b_other_in])) == 2
    # A COMPACT view (packed rows: pitch 3 x subscribed columns) is kept as it is.
    c = natural_item(W, H, 2, 0, 512, 512, 1024)
    c.in_pitch = 3 * (1024 - 510)
    assert rects(cover(pmb, [a, c])) == [(0, 512, 0, 512), (0, 512, 512, 1024)]
    # A gap, an overlap and mismatched row ranges do not merge.
    gap = natural_item(W, H, 2, 0, 512, 520, 1024)
    overlap = natural_item(W, H, 2, 0, 512, 500, 1024)
    taller = natural_item(W, H, 2, 0, 600, 512, 1024)
    for other in (gap, overlap, taller):
        assert len(cover(pmb, [a, other])) == 2


def test_l_shape_and_empty_items(pmb):
    W = H = 1024
    a = natural_item(W, H, 1, 0, 512, 0, 512)
    b = natural_item(W, H, 1, 0, 512, 512, 1024)
    c = natural_item(W, H, 1, 512, 1024, 0, 512)  # under a only: no rectangle with a + b
    e = natural_item(W, H, 1, 100, 100, 0, 512)   # empty
    assert rects(cover(pmb, [c, e, b, a])) == [(0, 512, 0, 1024), (512, 1024, 0, 512)]


def test_random_partitions_cover_every_pixel_once(pmb):
    rng = np.random.default_rng(1)
    for _ in range(30):
        W, H = int(rng.integers(40, 300)), int(rng.integers(40, 300))
        R = int(rng.integers(1, 9))
        cuts_r = sorted({0, H, *rng.integers(1, H, size=int(rng.integers(0, 6))).tolist()})
        cuts_c = sorted({0, W, *rng.integers(1, W, size=int(rng.integers(0, 6))).tolist()})
        items = [natural_item(W, H, R, r0, r1, c0, c1, runtime_origin=bool(rng.integers(0, 2)))
                 for r0, r1 in zip(cuts_r, cuts_r[1:]) for c0, c1 in zip(cuts_c, cuts_c[1:])]
        items = [items[i] for i in rng.permutation(len(items))]
        got = cover(pmb, items)
        assert 1 <= len(got) <= len(items)
        cnt = np.zeros((H, W), np.int32)
        for it in got:
            cnt[it.r0:it.r1, it.c0:it.c1] += 1
        assert (cnt == 1).all()
        assert rects(got) == [(0, H, 0, W)]
        # A random subset still covers exactly its own pixels.
        sub = items[: max(1, len(items) // 2)]
        want = np.zeros((H, W), np.int32)
        for it in sub:
            want[it.r0:it.r1, it.c0:it.c1] += 1
        cnt[:] = 0
        for it in cover(pmb, sub):
            cnt[it.r0:it.r1, it.c0:it.c1] += 1
        np.testing.assert_array_equal(cnt, want)


def test_cover_argument_checks(pmb):
    it = (capi.ImgfItem * 1)()
    out = (capi.ImgfItem * 1)()
    n = ctypes.c_int(0)
    assert pmb.pmb_image_filter_cover(it, 0, out, ctypes.byref(n)) == 7
    assert pmb.pmb_image_filter_cover(it, capi.PMB_IMGF_MAX_ITEMS + 1, out, ctypes.byref(n)) == 7
    assert pmb.pmb_image_filter_cover(it, 1, out, None) == 7
