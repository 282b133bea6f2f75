"""CPU tests of the C ABI library: it loads without a GPU, exports every
symbol include/pmb_capi.h declares, and rejects bad arguments before touching
the device."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

from conftest import ROOT, ptr


def header_functions() -> set[str]:
    names = set()
    with open(os.path.join(ROOT, "include", "pmb_capi.h")) as fh:
        text = fh.read()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(pmb_\w+)\s*\(", text, re.M):
        names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(pmb):
    from unicorn_b200 import capi

    declared = header_functions()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(pmb, name), f"libpmb.so does not export {name}"
    assert declared == set(capi.declared_symbols()), "capi.py bindings drift from the header"


def test_version_and_error_string(pmb):
    assert pmb.pmb_version().decode().count("_") == 2
    assert isinstance(pmb.pmb_last_error(), bytes)


def test_image_filter_argument_checks(pmb):
    from unicorn_b200 import capi

    f = np.zeros((32, 32), np.int8)
    dummy = ctypes.c_void_p(0x1000)
    # radius outside [1, 15]
    assert pmb.pmb_image_filter_full(dummy, dummy, 8, 8, ptr(f), 0, 0, None) == 7
    assert pmb.pmb_image_filter_full(dummy, dummy, 8, 8, ptr(f), 16, 0, None) == 7
    assert b"radius" in pmb.pmb_last_error()
    # bad mode
    assert pmb.pmb_image_filter_full(dummy, dummy, 8, 8, ptr(f), 1, 5, None) == 7
    # rectangle outside the image
    it = (capi.ImgfItem * 1)()
    it[0].in_ = it[0].out = 0x1000
    it[0].in_pitch = it[0].out_pitch = 24
    it[0].width, it[0].height = 8, 8
    it[0].r0, it[0].r1, it[0].c0, it[0].c1 = 0, 9, 0, 8
    assert pmb.pmb_image_filter(it, 1, ptr(f), 1, 0, None) == 7
    # input view that does not cover the subscription
    it[0].r1 = 8
    it[0].in_col0 = 3
    assert pmb.pmb_image_filter(it, 1, ptr(f), 1, 0, None) == 7
    assert b"input view" in pmb.pmb_last_error()
    # too many items
    assert pmb.pmb_image_filter(it, capi.PMB_IMGF_MAX_ITEMS + 1, ptr(f), 1, 0, None) == 7
