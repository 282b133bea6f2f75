"""The imageFiltering task over the pm:: API (unicorn_b200/serve/imgf_task):
submitted through pmSubmitTask with subscriptions restating the reference
app's imageFilterDataDistribution, run by the runtime's GPU stub (grouped
batched launches, staging and write-back), fetched with pmFetchMemory.  Its
output must equal the oracle's byte for byte, in both edge modes, with the
CUDA cache on and off, for images whose tiles are ragged at the edges."""
from __future__ import annotations

import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "unicorn_b200", "serve", "_build", "imgf_task")


@pytest.mark.parametrize("w,h,tile,radius,mode,cache,groups", [
    (700, 530, 128, 2, "clamp", 0, None),
    (700, 530, 128, 2, "wrap", 1, None),
    (1031, 517, 256, 3, "clamp", 0, "3"),
    (512, 512, 512, 1, "wrap", 0, "1"),
    (2048, 1536, 512, 2, "clamp", 0, "64"),
])
def test_imgf_task_matches_oracle(oracle, tmp_path, w, h, tile, radius, mode, cache, groups):
    env = dict(os.environ)
    if groups:
        env["PMB_BATCH_GROUPS"] = groups
    prefix = str(tmp_path / "imgf")
    p = subprocess.run([BIN, "--width", str(w), "--height", str(h), "--tile", str(tile), "--radius", str(radius),
                        "--mode", mode, "--cache", str(cache), "--steps", "2", "--warmup", "1", "--dump", prefix],
                       capture_output=True, text=True, timeout=300, env=env)
    assert p.returncode == 0, p.stderr
    rep = json.loads(p.stdout.strip().splitlines()[-1])
    assert rep["h2d_bytes_per_step"] >= 3 * w * h
    if cache == 0:
        assert rep["d2h_bytes_per_step"] == 3 * w * h
    img = np.fromfile(prefix + ".in", np.uint8)
    got = np.fromfile(prefix + ".out", np.uint8)
    filt = np.fromfile(prefix + ".filter", np.int8)
    expect = np.zeros_like(img)
    P = ctypes.c_void_p
    oracle.orc_image_filter(img.ctypes.data_as(P), expect.ctypes.data_as(P), w, h, radius, filt.ctypes.data_as(P),
                            1 if mode == "clamp" else 0, 0, h, 0, w)
    assert np.array_equal(got, expect), f"{int(np.count_nonzero(got != expect))} bytes differ"
