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


def test_reduce_argument_checks(pmb):
    """pmb_reduce_elementwise refuses bad operations, types, counts and
    misaligned pointers on the host (the fake device addresses are never
    dereferenced)."""
    srcs = (ctypes.c_void_p * 2)(0x1000, 0x2000)
    arr = ctypes.cast(srcs, ctypes.c_void_p)
    assert pmb.pmb_reduce_element_size(0) == 4 and pmb.pmb_reduce_element_size(5) == 8
    assert pmb.pmb_reduce_element_size(6) == 0
    assert pmb.pmb_reduce_elementwise(0, 0, None, arr, 2, 16, 1, None) == 7       # null destination
    assert pmb.pmb_reduce_elementwise(0, 0, 0x3000, arr, 0, 16, 1, None) == 7     # no sources
    assert pmb.pmb_reduce_elementwise(0, 9, 0x3000, arr, 2, 16, 1, None) == 7     # unknown type
    assert pmb.pmb_reduce_elementwise(0, 3, 0x3004, arr, 2, 16, 1, None) == 7     # 8-byte elements, 4-aligned
    bad = (ctypes.c_void_p * 2)(0x1000, 0x2002)
    assert pmb.pmb_reduce_elementwise(0, 0, 0x3000, ctypes.cast(bad, ctypes.c_void_p), 2, 16, 1, None) == 7
    assert b"aligned" in pmb.pmb_last_error()


def test_webdump_argument_checks(pmb):
    d = 0x1000
    # more pages than vertices; no slots; scratch too small
    assert pmb.pmb_csr_from_webdump(d, 10, 4, 5, 8, d, d, d, d, 1 << 30, None) == 7
    assert pmb.pmb_csr_from_webdump(d, 10, 0, 10, 8, d, d, d, d, 1 << 30, None) == 7
    need = pmb.pmb_webdump_csr_scratch_bytes(10, 10, 8)
    assert need > 0
    assert pmb.pmb_csr_from_webdump(d, 10, 4, 10, 8, d, d, d, d, need - 1, None) == 7
    assert pmb.pmb_csr_from_webdump(None, 10, 4, 10, 8, d, d, d, d, need, None) == 7
    # push: null output, no vertices
    assert pmb.pmb_webdump_push(d, 10, 4, None, 1.0, 0.85, None, 10, None, None) == 7
    assert pmb.pmb_webdump_push(d, 10, 4, None, 1.0, 0.85, d, 0, None, None) == 7
