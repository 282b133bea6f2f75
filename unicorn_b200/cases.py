"""Single kernel cases for profiling: `python -m unicorn_b200.cases <case> [size]`.

Each case builds seeded inputs on cuda:0, runs the operation once to warm up
and once more, synchronises and prints one line.  The second run is the one a
profiler capture selects (`ncu -k <kernel> -s <launches of the first run> -c 1`).

cases:
  gemm  N     C = A*B, N x N x N fp32 through the BF16x3 tcgen05 kernel
  lu    N     blocked LU of an N x N diagonally dominant matrix
  sort  N     8-bit LSD radix sort of N uint32 keys
  scan  N     inclusive uint32 -> uint64 scan of N elements
  imgf  W     W x W RGB image, 5x5 filter, 256-item batched launch
"""
from __future__ import annotations

import sys


def main(argv):
    import torch

    from unicorn_b200 import ops

    case = argv[1] if len(argv) > 1 else "gemm"
    g = torch.Generator(device="cuda").manual_seed(0)
    if case == "gemm":
        n = int(argv[2]) if len(argv) > 2 else 8192
        A = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
        B = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
        C, ws = ops.sgemm(A, B)
        C, ws = ops.sgemm(A, B, C, workspace=ws)
        out = float(C.abs().sum())
    elif case == "lu":
        n = int(argv[2]) if len(argv) > 2 else 4096
        A0 = (torch.rand(n, n, device="cuda", generator=g) * 2 - 1) + n * torch.eye(n, device="cuda")
        A = A0.clone()
        ops.lu_decompose(A)
        A = A0.clone()
        ops.lu_decompose(A)
        out = float(A.abs().sum())
    elif case in ("sort", "scan"):
        n = int(argv[2]) if len(argv) > 2 else 1 << 26
        keys = torch.randint(0, 2**32, (n,), dtype=torch.int64, device="cuda", generator=g).to(torch.uint32)
        if case == "sort":
            k = keys.clone()
            ops.radix_sort_u32(k)
            k = keys.clone()
            ops.radix_sort_u32(k)
            out = int(k[n // 2].item())
        else:
            y, scr = ops.inclusive_scan_u32_u64(keys)
            y, scr = ops.inclusive_scan_u32_u64(keys, y, scr)
            out = int(y[-1].item())
    elif case == "imgf":
        import numpy as np

        from unicorn_b200 import capi

        w = int(argv[2]) if len(argv) > 2 else 8192
        img = torch.randint(0, 256, (3 * w * w,), dtype=torch.uint8, device="cuda", generator=g)
        res = torch.empty_like(img)
        filt = np.random.default_rng(0).integers(-4, 5, size=(5, 5)).astype(np.int32)
        t = 512
        items = [(r, min(r + t, w), c, min(c + t, w)) for r in range(0, w, t) for c in range(0, w, t)]
        for _ in range(2):
            ops.image_filter(img, res, w, w, filt, mode=capi.PMB_IMGF_CLAMP, items=items)
        out = int(res.sum().item())
    else:
        raise SystemExit(__doc__)
    torch.cuda.synchronize()
    print(case, out)


if __name__ == "__main__":
    main(sys.argv)
