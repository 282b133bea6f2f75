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


def radix_sort_pairs_u32(d_keys, d_vals, begin_bit: int = 0, end_bit: int = 32, bits: int = 8, stream=None):
    """Stable in-place key-value sort (uint32 keys and values, int32 storage)."""
    import torch

    n = d_keys.numel()
    k_alt, v_alt = torch.empty_like(d_keys), torch.empty_like(d_vals)
    scratch = _scratch(capi.lib().pmb_radix_sort_scratch_bytes(n, bits))
    capi.check(capi.lib().pmb_radix_sort_pairs_u32(_dev_ptr(d_keys), _dev_ptr(k_alt), _dev_ptr(d_vals),
                                                   _dev_ptr(v_alt), n, begin_bit, end_bit, bits, _dev_ptr(scratch),
                                                   scratch.numel(), _stream_ptr(stream)))
    return d_keys, d_vals


def rmat_edges(seed: int, scale: int, n_edges: int, a=0.57, b=0.19, c=0.19, stream=None):
    import torch

    src = torch.empty(max(n_edges, 1), dtype=torch.int32, device="cuda")
    dst = torch.empty(max(n_edges, 1), dtype=torch.int32, device="cuda")
    capi.check(capi.lib().pmb_rmat_edges(seed, scale, n_edges, a, b, c, _dev_ptr(src), _dev_ptr(dst),
                                         _stream_ptr(stream)))
    return src[:n_edges], dst[:n_edges]


class CsrGraph:
    """Device CSR by destination plus the PageRank slice plan."""

    def __init__(self, d_src, d_dst, n_vertices: int, stream=None):
        import torch

        L = capi.lib()
        E = d_src.numel()
        self.n, self.e = n_vertices, E
        self.row_ptr = torch.empty(n_vertices + 1, dtype=torch.int32, device="cuda")
        self.col = torch.empty(max(E, 1), dtype=torch.int32, device="cuda")
        self.outdeg = torch.empty(n_vertices, dtype=torch.int32, device="cuda")
        scratch = self.csr_scratch = _scratch(L.pmb_csr_scratch_bytes(n_vertices, E))
        src = d_src if E else torch.zeros(1, dtype=torch.int32, device="cuda")
        dst = d_dst if E else torch.zeros(1, dtype=torch.int32, device="cuda")
        capi.check(L.pmb_csr_by_destination(_dev_ptr(src), _dev_ptr(dst), n_vertices, E, _dev_ptr(self.row_ptr),
                                            _dev_ptr(self.col), _dev_ptr(self.outdeg), _dev_ptr(scratch),
                                            scratch.numel(), _stream_ptr(stream)))
        self.plan = _scratch(L.pmb_pagerank_plan_bytes(n_vertices, E))
        capi.check(L.pmb_pagerank_plan(_dev_ptr(self.row_ptr), n_vertices, E, _dev_ptr(self.plan), self.plan.numel(),
                                       _stream_ptr(stream)))
        self.work = _scratch(L.pmb_pagerank_work_bytes(n_vertices, E))

    def build_error(self) -> int:
        """Error word of the CSR build (bit 2: an edge named a vertex >= n)."""
        return scratch_error(self.csr_scratch)

    def pagerank(self, rank_in, iterations: int, damping: float = 0.85, rank_out=None, stream=None):
        import torch

        if rank_out is None:
            rank_out = torch.empty_like(rank_in)
        capi.check(capi.lib().pmb_pagerank(_dev_ptr(self.row_ptr), _dev_ptr(self.col), _dev_ptr(self.outdeg), self.n,
                                           self.e, _dev_ptr(self.plan), damping, iterations, _dev_ptr(rank_in),
                                           _dev_ptr(rank_out), _dev_ptr(self.work), self.work.numel(),
                                           _stream_ptr(stream)))
        return rank_out


def sgemm(A, B, C=None, alpha: float = 1.0, beta: float = 0.0, plain: bool = False, workspace=None, stream=None):
    """Row-major fp32 C = alpha*A@B + beta*C on CUDA tensors (2-D, unit inner stride).

    plain=False: BF16x3 tcgen05 kernel; plain=True: FP32 SIMT kernel.
    Returns (C, workspace).
    """
    import torch

    M, K = A.shape
    K2, N = B.shape
    if K != K2:
        raise ValueError("inner dimensions differ")
    if C is None:
        C = torch.zeros(M, N, dtype=torch.float32, device=A.device)
    for t in (A, B, C):
        if t.dtype != torch.float32 or not t.is_cuda or t.stride(1) != 1:
            raise ValueError("fp32 CUDA matrices with unit column stride expected")
    L = capi.lib()
    if plain:
        capi.check(L.pmb_sgemm_plain(M, N, K, alpha, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), beta,
                                     C.data_ptr(), C.stride(0), _stream_ptr(stream)))
        return C, None
    need = L.pmb_gemm_workspace_bytes(M, N, K)
    if workspace is None or workspace.numel() < need:
        workspace = _scratch(need)
    capi.check(L.pmb_sgemm_bf16x3(M, N, K, alpha, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), beta,
                                  C.data_ptr(), C.stride(0), workspace.data_ptr(), workspace.numel(),
                                  _stream_ptr(stream)))
    return C, workspace


def sgemm_grouped(products, workspace=None, stream=None):
    """Several row-major fp32 products C = alpha*A@B + beta*C in one grouped
    BF16x3 call.  products: list of (A, B, C, alpha, beta) CUDA tensors /
    floats (2-D, unit column stride).  Returns the workspace."""
    import torch

    arr = (capi.GemmProblem * len(products))()
    for i, (A, B, C, alpha, beta) in enumerate(products):
        for t in (A, B, C):
            if t.dtype != torch.float32 or not t.is_cuda or t.stride(1) != 1:
                raise ValueError("fp32 CUDA matrices with unit column stride expected")
        M, K = A.shape
        K2, N = B.shape
        if K != K2 or tuple(C.shape) != (M, N):
            raise ValueError(f"product {i}: shapes {tuple(A.shape)} x {tuple(B.shape)} -> {tuple(C.shape)}")
        q = arr[i]
        q.M, q.N, q.K = M, N, K
        q.alpha, q.beta = alpha, beta
        q.A, q.lda, q.B, q.ldb, q.C, q.ldc = A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), C.data_ptr(), C.stride(0)
    L = capi.lib()
    need = L.pmb_gemm_grouped_workspace_bytes(arr, len(products))
    if workspace is None or workspace.numel() < need:
        workspace = _scratch(need)
    capi.check(L.pmb_sgemm_bf16x3_grouped(arr, len(products), workspace.data_ptr(), workspace.numel(),
                                          _stream_ptr(stream)))
    return workspace


def lu_decompose(d_A, nb: int = 64, plain: bool = False, workspace=None, stream=None):
    """In-place Crout LU of a square fp32 CUDA matrix stored column-major.

    d_A is a 2-D tensor whose memory holds the column-major matrix (i.e. the
    row-major transpose view).  Returns (d_A, workspace, flags) -- flags is the
    workspace flag word (1: pivoting would swap rows, 2: zero pivot).
    """
    n = d_A.shape[0]
    L = capi.lib()
    need = L.pmb_lu_workspace_bytes(n, nb)
    if workspace is None or workspace.numel() < need:
        workspace = _scratch(need)
    fn = L.pmb_lu_decompose_plain if plain else L.pmb_lu_decompose
    capi.check(fn(_dev_ptr(d_A), n, d_A.stride(0), nb, _dev_ptr(workspace), workspace.numel(), _stream_ptr(stream)))
    return d_A, workspace, scratch_error(workspace)


def lu_residual(d_A0, d_LU, stream=None) -> float:
    """||A0 - L*U||_F / ||A0||_F in FP64 (column-major storage for both)."""
    import torch

    n = d_A0.shape[0]
    sums = torch.zeros(2, dtype=torch.float64, device="cuda")
    capi.check(capi.lib().pmb_lu_residual_f64(_dev_ptr(d_A0), d_A0.stride(0), _dev_ptr(d_LU), d_LU.stride(0), n,
                                              _dev_ptr(sums), _stream_ptr(stream)))
    s = sums.cpu().numpy()
    return float(np.sqrt(s[0] / s[1])) if s[1] > 0 else 0.0


# pmReductionOpType / pmReductionDataType values (pmPublicUtilities.h)
REDUCE_OPS = ("ADD", "MIN", "MAX", "PRODUCT", "LOGICAL_AND", "BITWISE_AND", "LOGICAL_OR", "BITWISE_OR",
              "LOGICAL_XOR", "BITWISE_XOR")
REDUCE_TYPES = {"int32": 0, "uint32": 1, "int64": 2, "uint64": 3, "float32": 4, "float64": 5}


def reduce_elementwise(op: int, type_code: int, d_dst, srcs, count: int, init_from_first: bool = True,
                       stream=None):
    """Fold the device arrays `srcs` (in order) into d_dst over `count` elements
    with a built-in REDUCE_* operation (pmb_reduce_elementwise)."""
    ptrs = (ctypes.c_void_p * len(srcs))(*[_dev_ptr(s) for s in srcs])
    capi.check(capi.lib().pmb_reduce_elementwise(op, type_code, _dev_ptr(d_dst), ctypes.cast(ptrs, ctypes.c_void_p),
                                                 len(srcs), count, int(init_from_first), _stream_ptr(stream)))
    return d_dst
