"""CPU tests: the imageFilter oracle against the reference's own CPU callback.

The oracle (oracle/oracle.c orc_image_filter) is pinned against the golden
fixtures produced by the reference's imageFilter_cpu, and, where oracle/_ref
is built, against that callback directly on fresh seeded inputs.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import ROOT, ptr

GOLDEN = os.path.join(ROOT, "tests", "golden")


def run_oracle(oracle, img, W, H, R, f, mode, rect=None):
    out = np.zeros(H * W * 3, np.uint8)
    r0, r1, c0, c1 = rect or (0, H, 0, W)
    oracle.orc_image_filter(ptr(img), ptr(out), W, H, R, ptr(f), mode, r0, r1, c0, c1)
    return out


def golden_cases():
    z = np.load(os.path.join(GOLDEN, "imgf_golden.npz"))
    n = len([k for k in z.files if k.endswith("_meta")])
    for i in range(n):
        W, H, R, _ = (int(x) for x in z[f"c{i}_meta"])
        yield W, H, R, z[f"c{i}_in"], z[f"c{i}_filter"], z[f"c{i}_out"]


def test_oracle_matches_golden(oracle):
    count = 0
    for W, H, R, img, f, expect in golden_cases():
        got = run_oracle(oracle, img, W, H, R, f, 0)
        assert np.array_equal(got, expect), (W, H, R)
        count += 1
    assert count >= 6


@pytest.mark.parametrize("W,H,R,split", [(41, 29, 1, 0), (300, 260, 2, 4), (2100, 70, 3, 3), (9, 4, 6, 0)])
def test_oracle_matches_reference_callback(oracle, ref_imgf, W, H, R, split):
    rng = np.random.default_rng(W * 1000 + H + R)
    img = rng.integers(0, 256, size=H * W * 3, dtype=np.uint8)
    f = np.zeros((32, 32), np.int8)
    f[: 2 * R + 1, : 2 * R + 1] = rng.integers(-128, 128, size=(2 * R + 1, 2 * R + 1))
    expect = np.zeros_like(img)
    assert ref_imgf.ref_imgf_task(ptr(img), ptr(expect), W, H, R, ptr(f), 4, split) == 0
    assert np.array_equal(run_oracle(oracle, img, W, H, R, f, 0), expect)


def test_oracle_identity_filter_flips_rows_and_channels(oracle):
    # A centred delta filter copies the input: image row i is buffer row H-1-i,
    # output byte c comes from input byte 2-c (imageFiltering.cpp:438, :457-467).
    W, H, R = 7, 5, 1
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, size=(H, W, 3), dtype=np.uint8)
    f = np.zeros((32, 32), np.int8)
    f[1, 1] = 1
    for mode in (0, 1):
        out = run_oracle(oracle, img.reshape(-1), W, H, R, f, mode).reshape(H, W, 3)
        assert np.array_equal(out, img[::-1, :, ::-1])


def test_oracle_clamp_mode_saturates(oracle):
    W, H, R = 6, 4, 1
    img = np.full(H * W * 3, 200, np.uint8)
    f = np.zeros((32, 32), np.int8)
    f[:3, :3] = 1  # 9 * 200 = 1800 -> 255
    assert (run_oracle(oracle, img, W, H, R, f, 1) == 255).all()
    f[:3, :3] = -1
    assert (run_oracle(oracle, img, W, H, R, f, 1) == 0).all()
    # wrap mode keeps the low byte of the same sums: 1800 mod 256 = 8
    f[:3, :3] = 1
    assert (run_oracle(oracle, img, W, H, R, f, 0) == 1800 % 256).all()


def test_reference_subscription_geometry_fixture():
    # The reference's data-distribution callback subscribes, per subtask, the
    # output tile and the tile + halo rows/cols clamped to the image.  The
    # fixture (recorded from that callback) must agree with the closed form
    # the runtime's stub uses.
    with open(os.path.join(GOLDEN, "imgf_subscriptions.json")) as fh:
        shapes = json.load(fh)
    for sh in shapes:
        W, H, R, T = sh["W"], sh["H"], sh["R"], sh["tile_dim"]
        tpr = (W + T - 1) // T
        for sid, rec in enumerate(sh["subtasks"]):
            c0, r0 = (sid % tpr) * T, (sid // tpr) * T
            c1, r1 = min(c0 + T, W), min(r0 + T, H)
            fr, lr = max(0, r0 - R), min(H - 1, r1 - 1 + R)
            fc, lc = max(0, c0 - R), min(W - 1, c1 - 1 + R)
            row = 3 * W
            assert rec[0:4] == [(H - 1 - lr) * row + 3 * fc, 3 * (lc - fc + 1), row, lr - fr + 1]
            assert rec[4:8] == [r0 * row + 3 * c0, 3 * (c1 - c0), row, r1 - r0]
