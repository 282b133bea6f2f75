#!/usr/bin/env python
"""Benchmark of the B200 subtask path on the imageFiltering configuration.

Workload (one "step"): one imageFiltering task over a seeded synthetic
8192 x 8192 RGB image (bytes uniform in [0,255]), 5x5 integer filter with
weights uniform in [-4,4], output clamped to [0,255], split into 256 subtasks
of 512 x 512 output pixels (with their 2-pixel halos), all run in ONE launch of
the stencil kernel.  Input and output (201 MB each) exceed the 126 MB L2, so
no flush is needed between steps.

  value   : algorithmic bytes (read 3WH + write 3WH) per step / device time,
            inputs resident in HBM, CUDA events on the launching stream.
  e2e     : the same metric through the C ABI with host buffers: pinned host
            input -> H2D -> kernel -> D2H -> pinned host output, per step.
  roofline: the stencil kernel against the measured HBM copy bandwidth.
  cpu_baseline: the reference's own imageFilter_cpu (oracle/_ref, compiled
            from the reference sources) on the host cores, one worker per core.
  apps    : the other kernels of the path (radix sort, prefix sum, PageRank,
            GEMM, LU) on their configurations against their rooflines, each
            with a CPU figure (restated reference algorithm or BLAS-level
            restatement) on the same host.
  served_mix: the served mixed-size GEMM/LU stream over the pm:: API against
            the plain FP32 one-task-at-a-time form (unicorn_b200/serve).

`--impl reference` times that reference CPU implementation alone (the
reference has no runnable GPU path for this app: its texture-reference kernel
does not compile for CUDA 12).

Multi-GPU (torchrun): replicas only -- every rank filters its own image; value
is the bytes of all ranks over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = H = 8192
R = 2
TILE = 512
SEED = 3
ALG_BYTES = 2 * 3 * W * H  # 402,653,184
E2E_BANDS = 16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-apps", action="store_true", help="skip the per-app roofline measurements")
    ap.add_argument("--no-served", action="store_true", help="skip the served mixed-size task stream")
    ap.add_argument("--case", choices=["gemm", "lu", "sort", "scan", "imgf"],
                    help="profiling mode: run one kernel case twice (warm-up, then the captured run) and exit")
    ap.add_argument("--size", type=int, help="size of --case (N for gemm/lu, keys for sort/scan, W for imgf)")
    return ap.parse_args()


def run_case(case: str, size):
    """One kernel case on seeded inputs, run twice: the second run is the one
    a profiler capture selects (`ncu -k <kernel> -s <launches of the first
    run> -c 1`).  Prints one line and nothing is timed."""
    import torch

    from unicorn_b200 import capi, ops

    g = torch.Generator(device="cuda").manual_seed(0)
    if case == "gemm":
        n = size or 8192
        A = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
        B = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
        C, ws = ops.sgemm(A, B)
        C, ws = ops.sgemm(A, B, C, workspace=ws)
        out = float(C.abs().sum())
    elif case == "lu":
        n = size or 4096
        A0 = (torch.rand(n, n, device="cuda", generator=g) * 2 - 1) + n * torch.eye(n, device="cuda")
        for _ in range(2):
            A = A0.clone()
            ops.lu_decompose(A)
        out = float(A.abs().sum())
    elif case in ("sort", "scan"):
        n = size or 1 << 26
        keys = torch.randint(-2**31, 2**31, (n,), dtype=torch.int32, device="cuda", generator=g)
        if case == "sort":
            for _ in range(2):
                k = keys.clone()
                ops.radix_sort_u32(k)
            out = int(k[n // 2].item())
        else:
            y, scr = ops.inclusive_scan_u32_u64(keys)
            y, scr = ops.inclusive_scan_u32_u64(keys, y, scr)
            out = int(y[-1].item())
    else:  # imgf
        w = size or W
        img = torch.randint(0, 256, (3 * w * w,), dtype=torch.uint8, device="cuda", generator=g)
        res = torch.empty_like(img)
        filt = np.random.default_rng(0).integers(-4, 5, size=(5, 5)).astype(np.int32)
        items = [(r, min(r + TILE, w), c, min(c + TILE, w)) for r in range(0, w, TILE) for c in range(0, w, TILE)]
        for _ in range(2):
            ops.image_filter(img, res, w, w, filt, mode=capi.PMB_IMGF_CLAMP, items=items)
        out = int(res.sum().item())
    torch.cuda.synchronize()
    print(case, out)
    return 0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["bf16_tflops"])
    except Exception:
        return 1590.0


def profiled_traffic(kernel: str):
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of
    a kernel from one ncu capture, kept in profiles/dram_traffic.json."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as fh:
            return int(json.load(fh)[kernel]["bytes_per_launch"])
    except (OSError, KeyError, ValueError, TypeError):
        return None


def make_inputs():
    rng = np.random.default_rng(SEED)
    img = rng.integers(0, 256, size=H * W * 3, dtype=np.uint8)
    f = rng.integers(-4, 5, size=(2 * R + 1, 2 * R + 1)).astype(np.int8)
    return img, f


def tiles():
    return [(r, min(r + TILE, H), c, min(c + TILE, W)) for r in range(0, H, TILE) for c in range(0, W, TILE)]


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.lines:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(img, f, threads: int, min_seconds: float = 10.0, max_passes: int = 200):
    """Reference imageFilter_cpu over the whole 8192x8192 image, all threads.

    Repeats full passes until at least `min_seconds` of CPU work (a bounded
    sample of the same workload).  The reference computes the wrap (signed
    char) form; the cost per pixel is the same as the clamp form.
    """
    path = os.path.join(ROOT, "oracle", "_ref", "libref_imgf.so")
    if not os.path.exists(path):
        return None
    ref = ctypes.CDLL(path)
    fb = np.zeros((32, 32), np.int8)
    fb[: 2 * R + 1, : 2 * R + 1] = f
    out = np.zeros_like(img)
    P = ctypes.c_void_p
    split = max(1, (2 * threads + 15) // 16)  # 16 reference subtasks (TILE_DIM 2048), split over the cores
    passes, t0 = 0, time.perf_counter()
    while True:
        st = ref.ref_imgf_task(img.ctypes.data_as(P), out.ctypes.data_as(P), W, H, R, fb.ctypes.data_as(P), threads,
                               split)
        if st != 0:
            return None
        passes += 1
        dt = time.perf_counter() - t0
        if dt >= min_seconds or passes >= max_passes:
            break
    return {"value": round(ALG_BYTES * passes / dt / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": f"imageFilter_cpu (reference source, oracle/_ref) on the full {W}x{H} image, {passes} passes, "
                      f"{threads} worker threads, each of the 16 reference subtasks split {split} ways",
            "seconds": round(dt, 3)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    img, f = make_inputs()
    samples = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(img, f, threads, min_seconds=0.0, max_passes=1)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_imgf.so not built"}))
            return 0
        if i >= args.warmup:
            samples.append(r["value"])
    v = statistics.median(samples)
    line = {
        "impl": "reference", "metric": "imageFilter throughput (algorithmic bytes)", "value": v, "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ALG_BYTES / (v * 1e9) * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"imageFiltering {W}x{H} RGB, 5x5 filter, reference imageFilter_cpu (oracle/_ref), "
                               "one full-image pass per step", "threads": threads},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": "one full 8192x8192 pass per step"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _timed(torch, stream, fn, iters: int, warmup: int = 2) -> float:
    """Average ms of fn() over `iters`, CUDA events on `stream`."""
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(iters):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
    return a.elapsed_time(b) / iters


def app_measurements(torch, L, stream):
    """The other kernels of the path on their own configurations (sizes below),
    each against its roofline (measured peaks)."""
    from unicorn_b200 import capi, ops

    hbm, _ = peaks()
    bf16 = bf16_peak()
    sp = ctypes.c_void_p(stream.cuda_stream)
    res = {}
    with torch.cuda.stream(stream):
        # prefixSum + radixSort: 2^28 uint32 keys, seed 2
        n = 1 << 28
        g = torch.Generator(device="cuda").manual_seed(2)
        keys = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda", generator=g)
        work = keys.clone()
        alt = torch.empty_like(keys)
        ss = ops._scratch(L.pmb_radix_sort_scratch_bytes(n, 8))
        out64 = torch.empty(n, dtype=torch.int64, device="cuda")
        sc = ops._scratch(L.pmb_scan_scratch_bytes(n))

        def sort_once():
            work.copy_(keys)
            capi.check(L.pmb_radix_sort_u32(work.data_ptr(), alt.data_ptr(), n, 0, 32, 8, ss.data_ptr(), ss.numel(), sp))

        def scan_once():
            capi.check(L.pmb_inclusive_scan_u32_u64(work.data_ptr(), out64.data_ptr(), n, sc.data_ptr(), sc.numel(),
                                                    sp))

        # Checked once, outside the timed regions: a figure whose output is
        # wrong is dropped.
        sort_once()
        scan_once()
        torch.cuda.synchronize()
        k64 = work.to(torch.int64) & 0xFFFFFFFF
        sort_ok = bool(torch.equal(k64, torch.sort(keys.to(torch.int64) & 0xFFFFFFFF).values))
        scan_ok = int(out64[0]) == int(k64[0]) and bool(torch.equal(out64[1:] - out64[:-1], k64[1:]))
        err = ctypes.c_uint32(0)
        capi.check(L.pmb_scratch_error(ss.data_ptr(), ctypes.byref(err)))
        sort_ok = sort_ok and err.value == 0
        capi.check(L.pmb_scratch_error(sc.data_ptr(), ctypes.byref(err)))
        scan_ok = scan_ok and err.value == 0
        del k64
        copy_ms = _timed(torch, stream, lambda: work.copy_(keys), 5)
        sort_ms = _timed(torch, stream, sort_once, 5) - copy_ms
        scan_ms = _timed(torch, stream, scan_once, 10)
        # Library datapoints on the same keys and device: torch.sort of the
        # keys as int64 (their uint32 values) and torch.cumsum to int64.
        k64 = keys.to(torch.int64) & 0xFFFFFFFF
        tsort_ms = _timed(torch, stream, lambda: torch.sort(k64), 3)
        tscan_ms = _timed(torch, stream, lambda: torch.cumsum(work, 0, dtype=torch.int64), 5)
        del k64
        res["radix_sort_2^28"] = (_hbm_entry(8 * 4 * n, sort_ms, hbm) if sort_ok
                                  else {"error": "sorted keys differ from torch.sort or a look-back gave up"})
        res["radix_sort_2^28"]["library_torch_sort_int64_ms"] = round(tsort_ms, 4)
        res["prefix_sum_2^28"] = (_hbm_entry(12 * n, scan_ms, hbm) if scan_ok
                                  else {"error": "scan differs from the exact consecutive-difference check"})
        res["prefix_sum_2^28"]["library_torch_cumsum_int64_ms"] = round(tscan_ms, 4)
        del keys, work, alt, ss, out64, sc
        # pageRank: R-MAT 2^22 / 2^26, seed 1, 20 iterations
        nv, ne = 1 << 22, 1 << 26
        s_, d_ = ops.rmat_edges(1, 22, ne)
        gph = ops.CsrGraph(s_, d_, nv)
        r0 = torch.full((nv,), 1.0 / nv, dtype=torch.float32, device="cuda")
        rout = torch.empty_like(r0)
        pr_ms = _timed(torch, stream, lambda: gph.pagerank(r0, 20, rank_out=rout), 3) / 20
        res["pagerank_rmat22_per_iter"] = _hbm_entry(4 * (nv + 1) + 8 * ne + 8 * nv, pr_ms, hbm)
        del gph, s_, d_, r0, rout
        # GEMM: 1024^3 (16 subtasks of 256^2 as one GEMM) and 8192^3
        for dim in (1024, 8192):
            A = torch.rand(dim, dim, device="cuda", generator=g) * 2 - 1
            B = torch.rand(dim, dim, device="cuda", generator=g) * 2 - 1
            C = torch.empty(dim, dim, device="cuda")
            ws = ops._scratch(L.pmb_gemm_workspace_bytes(dim, dim, dim))
            it = 20 if dim <= 1024 else 5
            t = _timed(torch, stream, lambda: ops.sgemm(A, B, C, workspace=ws), it)
            tp = _timed(torch, stream, lambda: ops.sgemm(A, B, C, plain=True), 2 if dim > 1024 else it)
            torch.backends.cuda.matmul.allow_tf32 = False
            tc = _timed(torch, stream, lambda: torch.matmul(A, B, out=C), it)
            fl = 2.0 * dim ** 3
            res[f"gemm_bf16x3_{dim}"] = {
                "tflops": round(fl / t / 1e9, 1), "ms": round(t, 4),
                "roofline": {"bound": "tensor", "peak_fp32_equiv_tflops": round(bf16 / 3, 1),
                             "frac": round(fl / t / 1e9 / (bf16 / 3), 4),
                             "note": "3 bf16 MMAs per fp32 MAC; peak = measured bf16 cuBLAS / 3"},
                "plain_fp32_simt_tflops": round(fl / tp / 1e9, 2),
                "cublas_sgemm_fp32_tflops": round(fl / tc / 1e9, 2)}
            del A, B, C, ws
        # LU: n = 4096, diagonally dominant, nb = 64
        nl = 4096
        A0 = torch.rand(nl, nl, device="cuda", generator=g) * 2 - 1
        A0 += torch.eye(nl, device="cuda") * nl
        Aw = A0.clone()
        lws = ops._scratch(L.pmb_lu_workspace_bytes(nl, 64))

        def lu_once():
            Aw.copy_(A0)
            capi.check(L.pmb_lu_decompose(Aw.data_ptr(), nl, nl, 64, lws.data_ptr(), lws.numel(), sp))

        cp_ms = _timed(torch, stream, lambda: Aw.copy_(A0), 5)
        lu_ms = _timed(torch, stream, lu_once, 5) - cp_ms
        torch.cuda.synchronize()
        resid = ops.lu_residual(A0, Aw)
        res["lu_4096"] = {"gflops": round((2.0 / 3.0) * nl ** 3 / lu_ms / 1e6, 1), "ms": round(lu_ms, 3),
                          "residual_fro": resid, "launches": 3 * (nl // 64) - 2}
        del Aw, A0, lws
        # The LU trailing update alone at its largest step (rest = 4032, K = 64):
        # A22 -= L21*U12 streams A22 in and out (8 bytes per element); the split
        # pass over the two 4032 x 64 panels runs in the timed region too.
        m = nl - 64
        U = torch.rand(m, 64, device="cuda", generator=g) * 2 - 1
        V = torch.rand(64, m, device="cuda", generator=g) * 2 - 1
        C = torch.rand(m, m, device="cuda", generator=g) * 2 - 1
        uws = ops._scratch(L.pmb_gemm_workspace_bytes(m, m, 64))
        up_ms = _timed(torch, stream, lambda: ops.sgemm(U, V, C, -1.0, 1.0, workspace=uws), 20)
        res["lu_trailing_update_4032_k64"] = _hbm_entry(8 * m * m, up_ms, hbm)
        del U, V, C, uws
        # Subtask reduction (REDUCE_ADD, FLOATS): 8 subtask copies of 2^24
        # floats folded in order into the address space: 9 x 64 MiB moved.
        nr, ns = 1 << 24, 8
        copies = [torch.rand(nr, device="cuda", generator=g) for _ in range(ns)]
        dst = torch.empty(nr, device="cuda")
        red_ms = _timed(torch, stream, lambda: ops.reduce_elementwise(0, 4, dst, copies, nr, stream=stream), 10)
        res["subtask_reduce_add_f32_8x2^24"] = _hbm_entry(4 * nr * (ns + 1), red_ms, hbm)
        del copies, dst
        try:
            res.update(webdump_measurement(torch, L, stream, hbm))
        except Exception as e:  # a failed extra measurement must not lose the others
            res["webdump"] = {"error": f"{type(e).__name__}: {e}"}
    return res


def webdump_measurement(torch, L, stream, hbm: float, device: str = "cuda"):
    """The reference pageRank's own input format on the device: one push step
    (pmb_webdump_push) over 2^22 padded page records of 32 out-link slots
    (out-degrees uniform in [0, 32], so ~2^26 edges, the R-MAT 22 edge count),
    and the CSR build from the same records (pmb_csr_from_webdump)."""
    from unicorn_b200 import ops

    n, maxo = 1 << 22, 32
    g = torch.Generator(device=device).manual_seed(5)
    dump = torch.randint(1, n + 1, (n, maxo + 1), dtype=torch.int32, device=device, generator=g)
    counts = torch.randint(0, maxo + 1, (n,), dtype=torch.int32, device=device, generator=g)
    dump[:, 0] = counts
    edges = int(counts.sum().item())
    out = torch.empty(n, dtype=torch.float32, device=device)
    sp = ctypes.c_void_p(stream.cuda_stream)
    push_ms = _timed(torch, stream, lambda: capi_check(L.pmb_webdump_push(
        dump.data_ptr(), n, maxo, None, 1.0, 0.85, out.data_ptr(), n, None, sp)), 10)
    # algorithmic bytes: the records read once, the rank array zeroed and written
    push_bytes = 4 * n * (maxo + 1) + 4 * n
    res = {"webdump_push_2^22x32": dict(_hbm_entry(push_bytes, push_ms, hbm), edges=edges)}
    row_ptr = torch.empty(n + 1, dtype=torch.int32, device=device)
    col = torch.empty(max(edges, 1), dtype=torch.int32, device=device)
    deg = torch.empty(n, dtype=torch.int32, device=device)
    sc = ops._scratch(L.pmb_webdump_csr_scratch_bytes(n, n, edges)) if device == "cuda" else \
        torch.empty(L.pmb_webdump_csr_scratch_bytes(n, n, edges), dtype=torch.uint8)
    csr_ms = _timed(torch, stream, lambda: capi_check(L.pmb_csr_from_webdump(
        dump.data_ptr(), n, maxo, n, edges, row_ptr.data_ptr(), col.data_ptr(), deg.data_ptr(), sc.data_ptr(),
        sc.numel(), sp)), 3)
    res["csr_from_webdump_2^22x32"] = {"ms": round(csr_ms, 3), "edges": edges,
                                       "medges_per_s": round(edges / (csr_ms / 1e3) / 1e6, 1)}
    return res


def capi_check(st: int) -> None:
    from unicorn_b200 import capi

    capi.check(st)


def _oracle_lib():
    path = os.path.join(ROOT, "oracle", "liboracle.so")
    return ctypes.CDLL(path) if os.path.exists(path) else None


def _cpu_entry(value, unit, cores, kind, sample, seconds):
    return {"value": round(value, 3), "unit": unit, "cores": cores, "kind": kind, "sample": sample,
            "seconds": round(seconds, 3)}


def _reference_lib(name: str):
    path = os.path.join(ROOT, "oracle", "_ref", name)
    return ctypes.CDLL(path) if os.path.exists(path) else None


def reduce_cpu_baseline(orc, ref=None, nr: int = 1 << 24, ns: int = 8):
    """The reference's host fold (pmReducer::ReduceMemories REDUCE_ADD over
    FLOATS: the reference's own function from oracle/_ref/libref_reduce.so
    when given, else its restatement in oracle/oracle.c) on the same 8 copies
    of 2^24 floats: copy k folded into copy 0 for k = 1..7, one thread (the
    reference's loop is OpenMP-parallel only when built with
    USE_OMP_FOR_REDUCTION)."""
    P = ctypes.c_void_p
    rng = np.random.default_rng(4)
    copies = [rng.random(nr, dtype=np.float32) for _ in range(ns)]
    t0 = time.perf_counter()
    for k in range(1, ns):
        a, b = copies[0].ctypes.data_as(P), copies[k].ctypes.data_as(P)
        if ref is not None:
            ref.ref_reduce_memories(0, 4, a, b, ctypes.c_size_t(nr))
        else:
            orc.orc_reduce_fold(0, 4, a, b, ctypes.c_size_t(nr))
    dt = time.perf_counter() - t0
    what = ("pmReducer::ReduceMemories REDUCE_ADD (the reference's own, oracle/_ref)" if ref is not None else
            "pmReducer::ReduceMemories REDUCE_ADD restated (oracle/oracle.c)")
    return _cpu_entry(4.0 * nr * (ns + 1) / dt / 1e9, "GB/s", 1, "reference" if ref is not None else "port",
                      f"{what}, 8 copies of 2^24 floats folded pairwise into the first, one thread", dt)


def scan_sort_reference_baselines(res) -> bool:
    """Radix-sort and prefix-sum CPU figures from the reference's own serial
    functions (oracle/_ref/libref_scan_sort.so: serialLsbRadixSort with its
    4-bit digits in 8 rounds, serialPrefixSum over int32), one thread as the
    reference's per-subtask callbacks run, on bounded samples; rates in the
    configurations' algorithmic bytes (sort 32 B per key over 4 passes of
    8-bit digits, scan 12 B per element).  False when the library is absent."""
    ref = _reference_lib("libref_scan_sort.so")
    if ref is None:
        return False
    P, U = ctypes.c_void_p, ctypes.c_uint
    rng = np.random.default_rng(2)
    n = 1 << 24
    keys = rng.integers(0, 2**32, n, dtype=np.uint32)
    out = np.empty_like(keys)
    for _ in range(2):  # the first call faults the output pages in; time the second
        t0 = time.perf_counter()
        ref.ref_serial_lsb_radix_sort_u32(keys.ctypes.data_as(P), out.ctypes.data_as(P), U(n),
                                          ref.ref_radix_total_rounds())
        dt = time.perf_counter() - t0
    entries = {"radix_sort_2^28": _cpu_entry(
        32.0 * n / dt / 1e9, "GB/s", 1, "reference", "serialLsbRadixSort (the reference's own, oracle/_ref), "
        "4-bit digits x 8 rounds, 2^24 keys, one thread (the reference's per-subtask CPU sort)", dt)}
    m = 1 << 26
    vals = rng.integers(0, 16, m, dtype=np.int32)  # int32, the reference's type: sums stay below 2^31
    outv = np.empty_like(vals)
    for _ in range(2):
        t0 = time.perf_counter()
        ref.ref_serial_prefix_sum_i32(vals.ctypes.data_as(P), outv.ctypes.data_as(P), U(m))
        dt = time.perf_counter() - t0
    entries["prefix_sum_2^28"] = _cpu_entry(
        12.0 * m / dt / 1e9, "GB/s", 1, "reference", "serialPrefixSum (the reference's own, oracle/_ref, int32), "
        "2^26 elements, one thread", dt)
    for key, e in entries.items():
        if key in res:
            res[key]["cpu_baseline"] = e
    return True


def app_cpu_baselines(torch, res):
    """CPU figures next to each app kernel, on the box's host cores: the
    restated reference algorithms of oracle/ (bounded samples of the same
    workloads) and, for GEMM/LU, the reference's BLAS-level algorithm on the
    CBLAS that numpy ships (the reference calls cblas_sgemm/strsm/sscal/sger)."""
    from unicorn_b200 import ops

    orc = _oracle_lib()
    P = ctypes.c_void_p
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(2)
    if orc is not None and not scan_sort_reference_baselines(res):
        n = 1 << 24
        keys = rng.integers(0, 2**32, n, dtype=np.uint32)
        tmp = np.ones_like(keys)  # touched, so page faults stay out of the timed call
        t0 = time.perf_counter()
        orc.orc_radix_sort_u32(keys.ctypes.data_as(P), tmp.ctypes.data_as(P), ctypes.c_size_t(n), 0, 32, 8)
        dt = time.perf_counter() - t0
        res["radix_sort_2^28"]["cpu_baseline"] = _cpu_entry(
            32.0 * n / dt / 1e9, "GB/s", 1, "port", "serialRadixSortRound restated (oracle/oracle.c), 8-bit digits, "
            "2^24 keys, one thread (the reference's per-subtask CPU sort)", dt)
        vals = rng.integers(0, 2**32, 1 << 26, dtype=np.uint32)
        outv = np.ones(vals.size, np.uint64)
        t0 = time.perf_counter()
        orc.orc_prefix_sum_u32_u64(vals.ctypes.data_as(P), outv.ctypes.data_as(P), ctypes.c_size_t(vals.size))
        dt = time.perf_counter() - t0
        res["prefix_sum_2^28"]["cpu_baseline"] = _cpu_entry(
            12.0 * vals.size / dt / 1e9, "GB/s", 1, "port", "serialPrefixSum restated (oracle/oracle.c), 2^26 "
            "elements, one thread", dt)
        del keys, tmp, vals, outv
    if orc is not None:
        nv, ne = 1 << 22, 1 << 26
        s_, d_ = ops.rmat_edges(1, 22, ne)
        src = s_.cpu().numpy().view(np.uint32)
        dst = d_.cpu().numpy().view(np.uint32)
        order = np.argsort(src, kind="stable")
        src, dst = np.ascontiguousarray(src[order]), np.ascontiguousarray(dst[order])
        outdeg = np.bincount(src, minlength=nv).astype(np.uint32)
        outdeg[outdeg == 0] = 1
        r0 = np.full(nv, 1.0 / nv, np.float32)
        rout = np.empty_like(r0)
        t0 = time.perf_counter()
        orc.orc_pagerank_push_f32(src.ctypes.data_as(P), dst.ctypes.data_as(P), ctypes.c_uint64(ne), nv,
                                  outdeg.ctypes.data_as(P), 1, ctypes.c_float(0.85), r0.ctypes.data_as(P),
                                  rout.ctypes.data_as(P))
        dt = time.perf_counter() - t0
        res["pagerank_rmat22_per_iter"]["cpu_baseline"] = _cpu_entry(
            (4 * (nv + 1) + 8 * ne + 8 * nv) / dt / 1e9, "GB/s", 1, "port",
            "pageRank_cpu push arithmetic (oracle/oracle.c, bit-identical to the reference's), one iteration of "
            "the full R-MAT 2^22/2^26 graph, one thread", dt)
        del s_, d_, src, dst, order
        if "subtask_reduce_add_f32_8x2^24" in res:
            res["subtask_reduce_add_f32_8x2^24"]["cpu_baseline"] = reduce_cpu_baseline(
                orc, _reference_lib("libref_reduce.so"))
    if blas_reference_baselines(res, cores):
        return
    # Without oracle/_ref: the same BLAS calls on numpy's OpenBLAS.
    # GEMM: the reference CPU callback is cblas_sgemm (matrixMultiplyBlas.cpp:62-65).
    dim = 2048
    A = rng.random((dim, dim), dtype=np.float32) * 2 - 1
    B = rng.random((dim, dim), dtype=np.float32) * 2 - 1
    A @ B
    t0 = time.perf_counter()
    reps = 40
    for _ in range(reps):
        A @ B
    dt = (time.perf_counter() - t0) / reps
    for key in ("gemm_bf16x3_1024", "gemm_bf16x3_8192"):
        res[key]["cpu_baseline"] = _cpu_entry(2.0 * dim ** 3 / dt / 1e12, "TFLOP/s", cores, "port",
                                              f"cblas_sgemm via numpy's OpenBLAS, {dim}^3 fp32, all cores", dt)
    # LU: the reference's three stages per block (luDecomposition.cpp:116-125, 216-275, 301-347)
    # -- unblocked Crout of the diagonal block, two triangular solves, trailing sgemm -- on BLAS.
    import scipy.linalg as sla

    nl, nb = 2048, 256
    M = rng.random((nl, nl), dtype=np.float32) * 2 - 1 + nl * np.eye(nl, dtype=np.float32)
    a = np.asfortranarray(M)
    t0 = time.perf_counter()
    for k0 in range(0, nl, nb):
        k1 = min(nl, k0 + nb)
        d = a[k0:k1, k0:k1]
        for i in range(k1 - k0 - 1):
            d[i, i + 1:] /= d[i, i]
            d[i + 1:, i + 1:] -= np.outer(d[i + 1:, i], d[i, i + 1:])
        if k1 < nl:
            a[k0:k1, k1:] = sla.solve_triangular(np.tril(d), a[k0:k1, k1:], lower=True, check_finite=False)
            a[k1:, k0:k1] = sla.solve_triangular(np.triu(d, 1) + np.eye(k1 - k0, dtype=np.float32),
                                                 a[k1:, k0:k1].T, trans="T", lower=False, unit_diagonal=True,
                                                 check_finite=False).T
            a[k1:, k1:] -= a[k1:, k0:k1] @ a[k0:k1, k1:]
    dt = time.perf_counter() - t0
    res["lu_4096"]["cpu_baseline"] = _cpu_entry(
        (2.0 / 3.0) * nl ** 3 / dt / 1e9, "GFLOP/s", cores, "port",
        f"blocked Crout LU n={nl}, nb={nb}: the reference's 3 stages on numpy/scipy BLAS, all cores", dt)


def _time_reps(fn, min_seconds: float):
    """Seconds per call of fn, over at least min_seconds (one untimed call first)."""
    fn()
    reps, t0 = 0, time.perf_counter()
    while True:
        fn()
        reps += 1
        dt = time.perf_counter() - t0
        if dt >= min_seconds:
            return dt / reps


def blas_reference_baselines(res, cores: int, min_seconds: float = 2.0) -> bool:
    """GEMM and LU CPU figures from the reference's own CPU callbacks,
    compiled unchanged over numpy's OpenBLAS (oracle/_ref/libref_mm.so,
    libref_lu.so), all host cores through the BLAS threads:
    * gemm 1024: the task of 16 subtasks of 256 x 256 (matrixMultiply_cpu),
      fp32 U[-1,1] from seed 0 -- the reference's CPU-runnable configuration;
    * gemm 8192: a bounded sample, the 4096 task in the reference's own
      2048 x 2048 blocks (4 subtasks);
    * LU 4096: the app's LU_DECOMPOSE / HORZ_VERT_COMP / DIAGONAL_COMP sequence
      at its BLOCK_DIM 2048 on a diagonally dominant matrix (fresh copy per
      run, copy time excluded).
    Returns False (and sets nothing) when the libraries are absent."""
    mm_path = os.path.join(ROOT, "oracle", "_ref", "libref_mm.so")
    lu_path = os.path.join(ROOT, "oracle", "_ref", "libref_lu.so")
    if not (os.path.exists(mm_path) and os.path.exists(lu_path)):
        return False
    mm, lu = ctypes.CDLL(mm_path), ctypes.CDLL(lu_path)
    P, U = ctypes.c_void_p, ctypes.c_ulong
    entries = {}
    for key, n, block, seed in (("gemm_bf16x3_1024", 1024, 256, 0), ("gemm_bf16x3_8192", 4096, 2048, 1)):
        rng = np.random.default_rng(seed)
        a = rng.uniform(-1, 1, (n, n)).astype(np.float32)
        b = rng.uniform(-1, 1, (n, n)).astype(np.float32)
        c = np.empty_like(a)
        args = (a.ctypes.data_as(P), b.ctypes.data_as(P), c.ctypes.data_as(P), U(n), U(block))

        def run(args=args):
            if mm.ref_mm_task(*args) != 0:
                raise RuntimeError("reference matrixMultiply task failed")

        dt = _time_reps(run, min_seconds)
        entries[key] = _cpu_entry(2.0 * n ** 3 / dt / 1e12, "TFLOP/s", cores, "reference",
                                  f"reference matrixMultiply_cpu (oracle/_ref), {n}^2 fp32 in "
                                  f"{(n // block) ** 2} subtasks of {block}^2, all cores (BLAS threads)", dt)
    nl = 4096
    rng = np.random.default_rng(5)
    a0 = rng.uniform(-1, 1, (nl, nl)).astype(np.float32)
    a0[np.arange(nl), np.arange(nl)] += nl
    work = np.empty_like(a0)
    total, runs = 0.0, 0
    while total < min_seconds or runs < 2:
        np.copyto(work, a0)
        t0 = time.perf_counter()
        if lu.ref_lu_blocked(work.ctypes.data_as(P), U(nl)) != 0:
            raise RuntimeError("reference blocked LU failed")
        total += time.perf_counter() - t0
        runs += 1
    dt = total / runs
    entries["lu_4096"] = _cpu_entry(
        (2.0 / 3.0) * nl ** 3 / dt / 1e9, "GFLOP/s", cores, "reference",
        f"reference luDecomposition stages (oracle/_ref), n={nl} in blocks of 2048, all cores (BLAS threads)", dt)
    for key, e in entries.items():
        if key in res:
            res[key]["cpu_baseline"] = e
    return True


SERVED_BIN = os.path.join(ROOT, "unicorn_b200", "serve", "_build", "served_mix")
IMGF_TASK_BIN = os.path.join(ROOT, "unicorn_b200", "serve", "_build", "imgf_task")
SERVED_TASKS = 2000


def imgf_task_e2e(steps: int, warmup: int, device: int):
    """The imageFiltering configuration as a pm:: API task (pmSubmitTask of
    256 subtasks with their subscriptions, the runtime's GPU stub, result
    fetched to host memory), timed per step on the host clock in its own
    process on `device`."""
    if not os.path.exists(IMGF_TASK_BIN):
        return {"error": "imgf_task not built (make -C unicorn_b200/serve)"}
    env = dict(os.environ, PMB_DEVICE=str(device))
    p = subprocess.run(
        [IMGF_TASK_BIN, *map(str, ["--width", W, "--height", H, "--tile", TILE, "--radius", R, "--mode", "clamp",
                                   "--steps", steps, "--warmup", warmup, "--cache", 0, "--seed", SEED])],
        capture_output=True, text=True, timeout=600, env=env)
    lines = p.stdout.strip().splitlines()
    if p.returncode != 0 or not lines:
        return {"error": f"imgf_task exited {p.returncode}: {(p.stderr or p.stdout)[-300:]}"}
    return json.loads(lines[-1])


def _served_run(args):
    p = subprocess.run([SERVED_BIN, *map(str, args)], capture_output=True, text=True, timeout=1200)
    lines = p.stdout.strip().splitlines()
    if p.returncode != 0 or not lines:
        return {"error": f"served_mix exited {p.returncode}: {(p.stderr or p.stdout)[-300:]}"}
    return json.loads(lines[-1])


def served_measurement():
    """Served mixed-size stream (2,000 GEMM/LU tasks over the pm:: API) against
    the plain FP32 one-task-at-a-time form: first with arrivals faster than
    either form can serve (throughput), then at 75 % of the served capacity
    (latency under load; the plain form is overloaded at that rate)."""
    if not os.path.exists(SERVED_BIN):
        return {"error": "served_mix not built (make -C unicorn_b200/serve)"}
    keep = ("tasks_per_s", "completed", "span_s", "p50_ms", "p99_ms", "gemm_p50_ms", "gemm_p99_ms", "lu_p50_ms",
            "lu_p99_ms", "max_gemm_rel_err", "max_lu_residual", "error")
    sat = _served_run(["--tasks", SERVED_TASKS, "--rate", 20000])
    if "error" in sat:
        return sat
    out = {"workload": sat["workload"], "gemm_gflop": sat["gemm_gflop"], "lu_gflop": sat["lu_gflop"],
           "result_bytes": sat["result_bytes"], "plain_form": sat["plain_gemm"] + " GEMM, FP32 SIMT blocked LU, "
           "one task at a time",
           "saturated": {"rate_per_s": sat["rate_per_s"], "served": {k: sat["served"][k] for k in keep},
                         "plain": {k: sat["plain"][k] for k in keep},
                         "served_over_plain_tasks_per_s": sat.get("served_over_plain"),
                         "alone_vs_mix": sat["served_alone_vs_mix"]}}
    rate = round(0.75 * sat["served"]["tasks_per_s"], 1)
    ld = _served_run(["--tasks", SERVED_TASKS, "--rate", rate, "--check", 4])
    if "error" not in ld:
        out["at_load"] = {"rate_per_s": rate, "served": {k: ld["served"][k] for k in keep},
                          "plain": {k: ld["plain"][k] for k in keep}}
    return out


class Ranks:
    """One process per GPU (torchrun): rank and world size from the
    environment, a barrier after the caller's device sync, the max of a float
    over ranks, and the whole-job rate.  NCCL on the GPU box; the CPU tests
    run the same code over gloo."""

    def __init__(self, backend: str = "nccl", device=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device
        self.dist = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            kw = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
            self.dist = dist

    def barrier(self, sync=None) -> None:
        if sync is not None:
            sync()
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.dist is None:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device if self.device is not None else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank: float, steps: int, max_ms: float) -> float:
        """Whole-job units per second, in 1e9 units (GB/s for bytes): every
        rank processes units_per_rank per step; max_ms is the slowest rank."""
        return self.world * units_per_rank * steps / (max_ms / 1e3) / 1e9

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def _hbm_entry(nbytes: int, ms: float, hbm: float):
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"gbs": round(gbs, 1), "ms": round(ms, 4), "algorithmic_bytes": nbytes,
            "roofline": {"bound": "hbm", "peak": hbm, "frac": round(gbs / hbm, 4)}}


def summarize(line):
    """Compact per-app figures: {app: [rate, unit, roofline frac, CPU value,
    library or plain-form figure]} plus the served stream and the e2e path."""
    out = {}
    apps = line.get("apps") or {}

    def cpu(v):
        c = v.get("cpu_baseline") or {}
        return c.get("value")

    for key, v in apps.items():
        if not isinstance(v, dict):
            continue
        if "error" in v:
            out[key] = "error"
        elif "gbs" in v:
            lib = v.get("library_torch_sort_int64_ms") or v.get("library_torch_cumsum_int64_ms")
            out[key] = [v["gbs"], "GB/s", v["roofline"]["frac"], cpu(v)] + ([f"torch {lib} ms"] if lib else [])
        elif "tflops" in v:
            out[key] = [v["tflops"], "TFLOP/s", v["roofline"]["frac"], cpu(v), f"cublas_sgemm {v['cublas_sgemm_fp32_tflops']}"]
        elif "gflops" in v:
            out[key] = [v["gflops"], "GFLOP/s", v.get("ms"), cpu(v), f"resid {v.get('residual_fro')}"]
        elif "medges_per_s" in v:
            out[key] = [v["medges_per_s"], "Medges/s"]
    sm = line.get("served_mix") or {}
    sat = sm.get("saturated")
    if sat:
        out["served"] = {"tasks_per_s": sat["served"]["tasks_per_s"], "plain": sat["plain"]["tasks_per_s"],
                         "x": sat.get("served_over_plain_tasks_per_s"),
                         "alone_vs_mix": f"{sat['alone_vs_mix']['bit_identical']}/{sat['alone_vs_mix']['compared']}"}
        ld = sm.get("at_load")
        if ld:
            out["served"].update({"load_rate": ld["rate_per_s"], "p50_ms": ld["served"]["p50_ms"],
                                  "p99_ms": ld["served"]["p99_ms"]})
    elif sm:
        out["served"] = "error"
    e2e = line.get("e2e") or {}
    out["e2e"] = {"pm_api_gbs": e2e.get("value") if "pm_api_error" not in e2e else None,
                  "c_abi_gbs": (line.get("e2e_c_abi") or {}).get("value"),
                  "runtime_stub_ms": (e2e.get("runtime_per_task") or {}).get("stub_host_ms")}
    return out


def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.case:
        return run_case(args.case, args.size)

    import torch
    from unicorn_b200 import capi

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks("nccl", torch.device("cuda", local))
    world, rank = ranks.world, ranks.rank
    L = capi.lib()
    img, f = make_inputs()
    fb = np.zeros((32, 32), np.int8)
    fb[: 2 * R + 1, : 2 * R + 1] = f
    fp = fb.ctypes.data_as(ctypes.c_void_p)

    d_in = torch.from_numpy(img).cuda()
    d_out = torch.empty_like(d_in)
    rects = tiles()
    items = (capi.ImgfItem * len(rects))()
    for k, (r0, r1, c0, c1) in enumerate(rects):
        it = items[k]
        it.in_, it.out = d_in.data_ptr(), d_out.data_ptr()
        it.in_pitch = it.out_pitch = 3 * W
        it.width, it.height = W, H
        it.r0, it.r1, it.c0, it.c1 = r0, r1, c0, c1
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def step():
        capi.check(L.pmb_image_filter(items, len(rects), fp, R, capi.PMB_IMGF_CLAMP, sp))

    def barrier():
        ranks.barrier(torch.cuda.synchronize)

    max_over_ranks = ranks.max

    # ---- device-resident timing -----------------------------------------
    # The clock sampler starts first (its start-up pause would otherwise leave
    # the GPU idle right before the timed steps); then the warm-up steps, the
    # barrier + synchronize, and at once the timed steps.
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                step()
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        barrier()
    dev_ms = max_over_ranks(ev0.elapsed_time(ev1))
    ms_per_step = dev_ms / args.steps
    value = ranks.rate(ALG_BYTES, args.steps, dev_ms)
    kernel_gbs = ALG_BYTES / (ms_per_step / 1e3) / 1e9

    # ---- end to end through the pm:: API ------------------------------------
    # One imageFiltering task per step submitted with pmSubmitTask (256
    # subtasks, subscriptions as the reference app makes them), input staged
    # from the pinned host copy of its address space, output written back to
    # host memory and read there: host clock around each step.
    barrier()
    task = imgf_task_e2e(args.steps, args.warmup, local)
    e2e_ok = "error" not in task
    e2e_ms = max_over_ranks(task["ms_per_step"] * args.steps if e2e_ok else float("inf"))

    # ---- secondary: the C ABI host-buffer pipeline ---------------------------
    # pmb_image_filter_host: pinned host image in, pinned host image out; row
    # bands pipelined so uploads, the stencil and downloads overlap.
    h_in = torch.from_numpy(img).pin_memory()
    h_out = torch.empty(h_in.numel(), dtype=torch.uint8).pin_memory()

    def e2e_step():
        capi.check(L.pmb_image_filter_host(h_in.data_ptr(), h_out.data_ptr(), d_in.data_ptr(), d_out.data_ptr(), W, H,
                                           fp, R, capi.PMB_IMGF_CLAMP, E2E_BANDS, sp))

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    barrier()
    capi_ms = max_over_ranks(e0.elapsed_time(e1))
    capi_value = ranks.rate(ALG_BYTES, args.steps, capi_ms)
    capi_e2e = {"value": round(capi_value, 2), "unit": "GB/s", "h2d_bytes_per_step": 3 * W * H,
                "d2h_bytes_per_step": 3 * W * H,
                "path": f"C ABI pmb_image_filter_host, pinned host buffers, {E2E_BANDS} pipelined row bands"}
    if e2e_ok and e2e_ms != float("inf"):
        e2e = {"value": round(ranks.rate(ALG_BYTES, args.steps, e2e_ms), 2), "unit": "GB/s",
               "h2d_bytes_per_step": int(task["h2d_bytes_per_step"]),
               "d2h_bytes_per_step": int(task["d2h_bytes_per_step"]),
               "path": "pm:: API: pmSubmitTask of the imageFiltering task (256 subtasks, reference subscriptions, "
                       "cudaCacheEnabled false), pmWaitForTaskCompletion, pmFetchMemory + pmGetRawMemPtr of the "
                       "output; host clock per step (unicorn_b200/serve/imgf_task)",
               "ms_per_step": task["ms_per_step"], "ms_p50": task["ms_p50"],
               "runtime_per_task": {"stub_host_ms": task["stub_ms_per_task"],
                                    "callback_ms": task["callback_ms_per_task"],
                                    "batched_launches": task["batched_launches_per_task"]},
               "inputs": "same shapes and distributions as the device-resident run, generated in the task process"}
    else:
        e2e = dict(capi_e2e, pm_api_error=task.get("error", "a rank failed"))
    apps = None
    if rank == 0 and not args.no_apps:
        try:
            apps = app_measurements(torch, L, stream)
        except Exception as e:  # the extra kernels must not lose the headline line
            apps = {"error": f"{type(e).__name__}: {e}"}

    peak, peak_kind = peaks()
    line = {
        "metric": "imageFilter throughput (algorithmic bytes)", "value": round(value, 2), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "imageFiltering 8192x8192 RGB u8, 5x5 int filter [-4,4], clamp to [0,255], "
                               "256 subtasks of 512x512 (+2 px halo) in one launch",
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (201 MB in + 201 MB out)"},
        "roofline": {"bound": "hbm", "achieved": round(kernel_gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(kernel_gbs / peak, 4), "traffic": profiled_traffic("imgf_tc_kernel 8192x8192 5x5"),
                     "peak_source": f"{peak_kind} hbm_gbs (burst, kernel timed alone)"},
        "e2e": e2e,
        "e2e_c_abi": capi_e2e,
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    if apps is not None:
        if not args.no_cpu_baseline and "error" not in apps:
            try:
                app_cpu_baselines(torch, apps)
            except Exception as e:
                apps["cpu_baseline_error"] = f"{type(e).__name__}: {e}"
        line["apps"] = apps
    if rank == 0 and world == 1 and not args.no_served:
        torch.cuda.empty_cache()  # the served stream runs in its own process: leave it the device
        try:
            line["served_mix"] = served_measurement()
        except Exception as e:
            line["served_mix"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(img, f, os.cpu_count() or 1)
    # Last key of the line (so it survives a cut-off tail): one compact entry
    # per app kernel -- rate, roofline fraction, CPU baseline, library figure.
    line["summary"] = summarize(line)
    ranks.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
