"""ctypes binding of libpmb.so, the C ABI of the B200 subtask path.

Every function declared in include/pmb_capi.h is bound here with its exact
argument types.  Loading fails loudly (ImportError) when the library has not
been built: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpmb.so")

c_void_p = ctypes.c_void_p
c_int = ctypes.c_int
c_int64 = ctypes.c_int64
c_size_t = ctypes.c_size_t

PMB_SUCCESS = 0
PMB_INVALID_INDEX = 7
PMB_IMGF_WRAP = 0
PMB_IMGF_CLAMP = 1
PMB_IMGF_MAX_ITEMS = 256
PMB_IMGF_MAX_FILTER_DIM = 32
PMB_SCAN_NOALLOC_MAX_ELEMS = 1 << 30
PMB_BEYOND_LIMITS = 15
PMB_SIDE_LEFT, PMB_SIDE_RIGHT = 0, 1
PMB_FILL_LOWER, PMB_FILL_UPPER = 0, 1
PMB_DIAG_NON_UNIT, PMB_DIAG_UNIT = 0, 1


class PmbError(RuntimeError):
    """A libpmb.so call returned a non-zero pmStatus."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"pmStatus {status}: {msg}")
        self.status = status


class GemmProblem(ctypes.Structure):
    """Mirror of pmb_gemm_problem (include/pmb_capi.h)."""

    _fields_ = [
        ("M", ctypes.c_int32),
        ("N", ctypes.c_int32),
        ("K", ctypes.c_int32),
        ("alpha", ctypes.c_float),
        ("A", c_void_p),
        ("lda", c_int64),
        ("B", c_void_p),
        ("ldb", c_int64),
        ("beta", ctypes.c_float),
        ("C", c_void_p),
        ("ldc", c_int64),
    ]


class ImgfItem(ctypes.Structure):
    """Mirror of pmb_imgf_item (include/pmb_capi.h)."""

    _fields_ = [
        ("in_", c_void_p),
        ("out", c_void_p),
        ("in_pitch", c_int64),
        ("out_pitch", c_int64),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("in_row0", ctypes.c_int32),
        ("in_col0", ctypes.c_int32),
        ("out_row0", ctypes.c_int32),
        ("out_col0", ctypes.c_int32),
        ("r0", ctypes.c_int32),
        ("r1", ctypes.c_int32),
        ("c0", ctypes.c_int32),
        ("c1", ctypes.c_int32),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "pmb_last_error": (ctypes.c_char_p, []),
    "pmb_version": (ctypes.c_char_p, []),
    "pmb_device_supported": (c_int, [c_int]),
    "pmb_device_count": (c_int, [ctypes.POINTER(c_int)]),
    "pmb_set_device": (c_int, [c_int]),
    "pmb_device_properties": (c_int, [c_int, ctypes.c_char_p, c_size_t, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                      ctypes.POINTER(c_int)]),
    "pmb_mem_get_info": (c_int, [ctypes.POINTER(c_size_t), ctypes.POINTER(c_size_t)]),
    "pmb_malloc": (c_int, [ctypes.POINTER(c_void_p), c_size_t]),
    "pmb_free": (c_int, [c_void_p]),
    "pmb_malloc_async": (c_int, [ctypes.POINTER(c_void_p), c_size_t, c_void_p]),
    "pmb_free_async": (c_int, [c_void_p, c_void_p]),
    "pmb_host_alloc": (c_int, [ctypes.POINTER(c_void_p), c_size_t]),
    "pmb_host_free": (c_int, [c_void_p]),
    "pmb_stream_create": (c_int, [ctypes.POINTER(c_void_p)]),
    "pmb_stream_destroy": (c_int, [c_void_p]),
    "pmb_stream_synchronize": (c_int, [c_void_p]),
    "pmb_event_create": (c_int, [ctypes.POINTER(c_void_p), c_int]),
    "pmb_event_destroy": (c_int, [c_void_p]),
    "pmb_event_record": (c_int, [c_void_p, c_void_p]),
    "pmb_event_query": (c_int, [c_void_p]),
    "pmb_event_synchronize": (c_int, [c_void_p]),
    "pmb_event_elapsed_ms": (c_int, [c_void_p, c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "pmb_stream_wait_event": (c_int, [c_void_p, c_void_p]),
    "pmb_memcpy_async": (c_int, [c_void_p, c_void_p, c_size_t, c_int, c_void_p]),
    "pmb_memcpy2d_async": (c_int, [c_void_p, c_size_t, c_void_p, c_size_t, c_size_t, c_size_t, c_int, c_void_p]),
    "pmb_memset_async": (c_int, [c_void_p, c_int, c_size_t, c_void_p]),
    "pmb_launch_kernel": (c_int, [c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                  ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(c_void_p), c_void_p]),
    "pmb_device_synchronize": (c_int, []),
    "pmb_copy_ranges": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "pmb_mempool_retain": (c_int, [c_int]),
    "pmb_mempool_reserve": (c_int, [c_int, c_size_t, c_void_p]),
    "pmb_reduce_element_size": (c_size_t, [c_int]),
    "pmb_webdump_csr_scratch_bytes": (c_size_t, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]),
    "pmb_csr_from_webdump": (c_int, [c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                     c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "pmb_webdump_push": (c_int, [c_void_p, ctypes.c_uint32, ctypes.c_uint32, c_void_p, ctypes.c_float,
                                 ctypes.c_float, c_void_p, ctypes.c_uint32, c_void_p, c_void_p]),
    "pmb_reduce_elementwise": (c_int, [c_int, c_int, c_void_p, c_void_p, c_int, c_size_t, c_int, c_void_p]),
    "pmb_mempool_trim": (c_int, [c_int, c_size_t]),
    "pmb_mem_available": (c_int, [c_int, ctypes.POINTER(c_size_t)]),
    "pmb_graph_begin_capture": (c_int, [c_void_p]),
    "pmb_graph_end_capture": (c_int, [c_void_p, ctypes.POINTER(c_void_p)]),
    "pmb_graph_launch": (c_int, [c_void_p, c_void_p]),
    "pmb_graph_destroy": (c_int, [c_void_p]),
    "pmb_image_filter": (c_int, [ctypes.POINTER(ImgfItem), c_int, c_void_p, c_int, c_int, c_void_p]),
    "pmb_image_filter_full": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_int, c_void_p]),
    "pmb_image_filter_host": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_int,
                                      c_int, c_void_p]),
    "pmb_image_filter_error": (c_int, [c_int, ctypes.POINTER(ctypes.c_uint32)]),
    "pmb_image_filter_cover": (c_int, [ctypes.POINTER(ImgfItem), c_int, ctypes.POINTER(ImgfItem),
                                       ctypes.POINTER(c_int)]),
    "pmb_trsm_workspace_bytes": (c_size_t, [c_int, c_int, c_int]),
    "pmb_lu_refine_workspace_bytes": (c_size_t, [c_int]),
    "pmb_lu_solve_refined": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_int, c_void_p, c_void_p, c_int, c_void_p,
                                     c_void_p, c_size_t, c_void_p]),
    "pmb_trsm_f32": (c_int, [c_int, c_int, c_int, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                             c_size_t, c_void_p]),
    "pmb_image_filter_plain": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_int, c_void_p]),
    "pmb_sentinel_capacity_bytes": (c_size_t, [c_int, c_size_t]),
    "pmb_sentinel_scratch_bytes": (c_size_t, [c_int, c_size_t]),
    "pmb_sentinel_compress": (c_int, [c_int, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p]),
    "pmb_sentinel_compressed": (c_int, [c_int, c_size_t, ctypes.c_uint32]),
    "pmb_sentinel_expand": (c_int, [c_int, c_void_p, c_void_p, c_size_t]),
    "pmb_scan_scratch_bytes": (c_size_t, [c_size_t]),
    "pmb_inclusive_scan_u32_u64": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p]),
    "pmb_inclusive_scan_u32_u64_noalloc": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p]),
    "pmb_scan_noalloc_error": (c_int, [ctypes.POINTER(ctypes.c_uint32)]),
    "pmb_scratch_error": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_uint32)]),
    "pmb_radix_sort_scratch_bytes": (c_size_t, [c_size_t, c_int]),
    "pmb_radix_sort_histogram": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "pmb_add_u64_scalar": (c_int, [c_void_p, c_size_t, c_void_p, c_void_p]),
    "pmb_radix_sort_u32": (c_int, [c_void_p, c_void_p, c_size_t, c_int, c_int, c_int, c_void_p, c_size_t, c_void_p]),
    "pmb_radix_sort_pairs_u32": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_int, c_int, c_int,
                                         c_void_p, c_size_t, c_void_p]),
    "pmb_rmat_edges": (c_int, [ctypes.c_uint64, c_int, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, c_void_p, c_void_p, c_void_p]),
    "pmb_csr_scratch_bytes": (c_size_t, [ctypes.c_uint32, ctypes.c_uint64]),
    "pmb_csr_by_destination": (c_int, [c_void_p, c_void_p, ctypes.c_uint32, ctypes.c_uint64, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_size_t, c_void_p]),
    "pmb_pagerank_plan_bytes": (c_size_t, [ctypes.c_uint32, ctypes.c_uint64]),
    "pmb_pagerank_plan": (c_int, [c_void_p, ctypes.c_uint32, ctypes.c_uint64, c_void_p, c_size_t, c_void_p]),
    "pmb_pagerank_work_bytes": (c_size_t, [ctypes.c_uint32, ctypes.c_uint64]),
    "pmb_gemm_workspace_bytes": (c_size_t, [c_int, c_int, c_int]),
    "pmb_sgemm_bf16x3": (c_int, [c_int, c_int, c_int, ctypes.c_float, c_void_p, c_int64, c_void_p, c_int64,
                                 ctypes.c_float, c_void_p, c_int64, c_void_p, c_size_t, c_void_p]),
    "pmb_gemm_grouped_workspace_bytes": (c_size_t, [c_void_p, c_int]),
    "pmb_sgemm_bf16x3_grouped": (c_int, [c_void_p, c_int, c_void_p, c_size_t, c_void_p]),
    "pmb_sgemm_plain": (c_int, [c_int, c_int, c_int, ctypes.c_float, c_void_p, c_int64, c_void_p, c_int64,
                                ctypes.c_float, c_void_p, c_int64, c_void_p]),
    "pmb_lu_workspace_bytes": (c_size_t, [c_int, c_int]),
    "pmb_lu_decompose": (c_int, [c_void_p, c_int, c_int64, c_int, c_void_p, c_size_t, c_void_p]),
    "pmb_lu_decompose_plain": (c_int, [c_void_p, c_int, c_int64, c_int, c_void_p, c_size_t, c_void_p]),
    "pmb_lu_residual_f64": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_int, c_void_p, c_void_p]),
    "pmb_pagerank": (c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_uint32, ctypes.c_uint64, c_void_p,
                             ctypes.c_float, c_int, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libpmb.so once (raises ImportError if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `make -C unicorn_b200/csrc`")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(status: int) -> None:
    if status != PMB_SUCCESS:
        raise PmbError(status, lib().pmb_last_error().decode())


def declared_symbols() -> list[str]:
    return list(_SIGS)
