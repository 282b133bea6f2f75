"""Served mixed-size task stream (unicorn_b200/serve/served_mix) over the pm::
API: GEMM and LU tasks arriving as a Poisson stream, run concurrently by the
runtime (served form) and one at a time in FP32 (plain form).

The GPU tests run a small stream and check what the serving benchmark claims:
every task completes, each sampled result inside the mix is bit-identical to
the same task run alone, the split-precision results stay within 1e-5 of FP64
(GEMM relative Frobenius error, LU ||A - LU||_F / ||A||_F), and the plain FP32
results are reported beside them.
"""
from __future__ import annotations

import json
import os
import subprocess

import pytest

from conftest import ROOT

SERVE_DIR = os.path.join(ROOT, "unicorn_b200", "serve")
BIN = os.path.join(SERVE_DIR, "_build", "served_mix")

# Split precision must recover FP32 accuracy (stated tolerance vs FP64).
REL_TOL = 1e-5


@pytest.fixture(scope="module")
def served_bin():
    subprocess.run(["make", "-s", "-C", SERVE_DIR], check=True, stdout=subprocess.DEVNULL)
    return BIN


def run(cmd, timeout=900):
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    return p.returncode, p.stdout, p.stderr


def test_served_mix_rejects_bad_arguments(served_bin):
    rc, out, err = run([served_bin, "--gemm-max", "9000"])
    assert rc == 2 and "usage" in err
    rc, out, err = run([served_bin, "--bogus"])
    assert rc == 2


@pytest.mark.gpu
@pytest.mark.parametrize("plain_gemm", ["cublas", "simt"])
def test_served_mix_small_stream(served_bin, plain_gemm):
    rc, out, err = run([served_bin, "--tasks", "80", "--rate", "400", "--gemm-min", "64", "--gemm-max", "1024",
                        "--lu-min", "64", "--lu-max", "1024", "--warmup", "8", "--check", "12",
                        "--plain-gemm", plain_gemm])
    assert rc == 0, out + err
    r = json.loads(out.strip().splitlines()[-1])
    assert "error" not in r, r
    for form in ("served", "plain"):
        s = r[form]
        assert s["error"] == "", s
        assert s["completed"] == 80
        assert s["p99_ms"] >= s["p50_ms"] > 0
        assert len(s["checks"]) == 12
    assert r["served"]["max_gemm_rel_err"] <= REL_TOL
    assert r["served"]["max_lu_residual"] <= REL_TOL
    assert r["plain"]["max_gemm_rel_err"] <= REL_TOL
    assert r["plain"]["max_lu_residual"] <= REL_TOL
    a = r["served_alone_vs_mix"]
    assert a["compared"] == 12 and a["bit_identical"] == 12, a


@pytest.mark.gpu
def test_served_mix_admits_under_memory_pressure(served_bin):
    """Many large tasks at once with few slots: the runtime must queue them
    (admission) rather than fail, and results stay exact."""
    env = dict(os.environ, PMB_MAX_INFLIGHT="3", PMB_STREAMS="2")
    p = subprocess.run([served_bin, "--tasks", "24", "--rate", "0", "--gemm-min", "2048", "--gemm-max", "4096",
                        "--lu-min", "1024", "--lu-max", "2048", "--warmup", "2", "--check", "4", "--mode", "served"],
                       capture_output=True, text=True, timeout=900, env=env)
    assert p.returncode == 0, p.stdout + p.stderr
    r = json.loads(p.stdout.strip().splitlines()[-1])
    s = r["served"]
    assert s["error"] == "" and s["completed"] == 24, s
    assert s["max_gemm_rel_err"] <= REL_TOL and s["max_lu_residual"] <= REL_TOL
    assert r["served_alone_vs_mix"]["bit_identical"] == r["served_alone_vs_mix"]["compared"] == 4


@pytest.mark.gpu
def test_served_mix_concurrent_lu_stream_completes(served_bin):
    """Many LU tasks admitted at once: their block-step kernels from different
    tasks share the SMs (a trailing-update kernel variant that packed three
    CTAs per SM once stalled exactly this case).  Every task must finish,
    exact and bit-identical to its run alone."""
    p = subprocess.run([served_bin, "--tasks", "64", "--rate", "0", "--gemm-frac", "0", "--lu-min", "512",
                        "--lu-max", "4096", "--warmup", "64", "--check", "4", "--mode", "served"],
                       capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout + p.stderr
    r = json.loads(p.stdout.strip().splitlines()[-1])
    s = r["served"]
    assert s["error"] == "" and s["completed"] == 64, s
    assert s["max_lu_residual"] <= REL_TOL
    assert r["served_alone_vs_mix"]["bit_identical"] == r["served_alone_vs_mix"]["compared"] == 4
