"""Array-level wrappers over the C ABI for torch CUDA tensors.

Device memory and streams come from torch (plumbing only); every computation
runs in libpmb.so.  A tensor that is not on a CUDA device is rejected: there is
no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi


def _stream_ptr(stream) -> int:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _dev_ptr(t) -> int:
    if not t.is_cuda:
        raise ValueError("libpmb.so operates on CUDA tensors only (no CPU fallback)")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return int(t.data_ptr())


def filter_bytes(filt: np.ndarray) -> np.ndarray:
    """Embed a (2R+1)x(2R+1) int8 filter into the 32x32 layout of imageFilterTaskConf."""
    f = np.zeros((capi.PMB_IMGF_MAX_FILTER_DIM, capi.PMB_IMGF_MAX_FILTER_DIM), np.int8)
    k = filt.shape[0]
    f[:k, :k] = filt
    return f


def image_filter(d_in, d_out, width: int, height: int, filt: np.ndarray, mode: int = capi.PMB_IMGF_WRAP,
                 items=None, stream=None) -> None:
    """Filter the whole image (items=None) or a list of subtask rectangles.

    d_in / d_out: uint8 CUDA tensors with 3*W*H bytes (NATURAL views of the
    bottom-up input and top-down output address spaces).  items: optional list of
    (r0, r1, c0, c1) output rectangles run in one launch.
    """
    R = (filt.shape[0] - 1) // 2
    f = filter_bytes(filt)
    fp = f.ctypes.data_as(ctypes.c_void_p)
    L = capi.lib()
    if items is None:
        capi.check(L.pmb_image_filter_full(_dev_ptr(d_in), _dev_ptr(d_out), width, height, fp, R, mode,
                                           _stream_ptr(stream)))
        return
    arr = (capi.ImgfItem * len(items))()
    for k, (r0, r1, c0, c1) in enumerate(items):
        it = arr[k]
        it.in_ = _dev_ptr(d_in)
        it.out = _dev_ptr(d_out)
        it.in_pitch = it.out_pitch = 3 * width
        it.width, it.height = width, height
        it.in_row0 = it.in_col0 = it.out_row0 = it.out_col0 = 0
        it.r0, it.r1, it.c0, it.c1 = r0, r1, c0, c1
    capi.check(L.pmb_image_filter(arr, len(items), fp, R, mode, _stream_ptr(stream)))


def image_filter_plain(d_in, d_out, width: int, height: int, filt: np.ndarray,
                       mode: int = capi.PMB_IMGF_WRAP, stream=None) -> None:
    R = (filt.shape[0] - 1) // 2
    f = filter_bytes(filt)
    capi.check(capi.lib().pmb_image_filter_plain(_dev_ptr(d_in), _dev_ptr(d_out), width, height,
                                                 f.ctypes.data_as(ctypes.c_void_p), R, mode,
                                                 _stream_ptr(stream)))


def _scratch(nbytes: int):
    import torch

    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device="cuda")


def scratch_error(scratch) -> int:
    err = ctypes.c_uint32(0)
    capi.check(capi.lib().pmb_scratch_error(_dev_ptr(scratch), ctypes.byref(err)))
    return int(err.value)


def inclusive_scan_u32_u64(d_in, d_out=None, scratch=None, stream=None):
    """Inclusive 64-bit prefix sum of a uint32 CUDA tensor (int32/uint32 storage).

    Returns (d_out, scratch); d_out holds the 64-bit sums in int64 storage.
    """
    import torch

    n = d_in.numel()
    if d_out is None:
        d_out = torch.empty(n, dtype=torch.int64, device=d_in.device)
    need = capi.lib().pmb_scan_scratch_bytes(n)
    if scratch is None or scratch.numel() < need:
        scratch = _scratch(need)
    capi.check(capi.lib().pmb_inclusive_scan_u32_u64(_dev_ptr(d_in), _dev_ptr(d_out), n, _dev_ptr(scratch),
                                                     scratch.numel(), _stream_ptr(stream)))
    return d_out, scratch


def radix_sort_u32(d_keys, begin_bit: int = 0, end_bit: int = 32, bits: int = 8, d_alt=None, scratch=None,
                   stream=None):
    """Stable in-place LSD sort of a uint32 CUDA tensor (int32/uint32 storage)."""
    import torch

    n = d_keys.numel()
    if d_alt is None:
        d_alt = torch.empty_like(d_keys)
    need = capi.lib().pmb_radix_sort_scratch_bytes(n, bits)
    if scratch is None or scratch.numel() < need:
        scratch = _scratch(need)
    capi.check(capi.lib().pmb_radix_sort_u32(_dev_ptr(d_keys), _dev_ptr(d_alt), n, begin_bit, end_bit, bits,
                                             _dev_ptr(scratch), scratch.numel(), _stream_ptr(stream)))
    return d_keys, scratch
