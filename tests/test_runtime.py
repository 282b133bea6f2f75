"""pm:: runtime tests (libpmlib.so) through its public C++ API.

* tests/runtime/rt_selftest: our own driver of the API -- scattered
  subscriptions, NATURAL and COMPACT views, scratch buffers, launch
  configuration and reserved memory for an app-style subtask_gpu_cuda kernel,
  chained tasks that stay device-resident, write-through with the CUDA cache
  disabled, many tasks in flight vs alone, error returns and timeouts, and
  subtask reduction (every built-in REDUCE_* operation and data type, partial
  and scattered writes, the app's own callbacks) and ordered redistribution
  (pmRedistributeData / pmGetRedistributionMetadata, radixSort's bucket
  pattern) on the CPU and on the GPU.
* oracle/_ref/imageFiltering_b200.exe: the reference's own imageFiltering app
  and harness (imageFiltering.cpp + commonAPI.cpp, unchanged) linked against
  this runtime and the B200 GPU callbacks; it checks itself against its serial
  CPU implementation and prints "Serial Comparison Test Passed".
* oracle/_ref/matrixMultiplyBlas_b200.exe and luDecomposition_cpu.exe: the
  reference's BLAS apps (matrixMultiplyBlas.cpp, luDecomposition.cpp +
  commonAPI.cpp, unchanged, CBLAS through the shim on numpy's OpenBLAS) on the
  runtime's CPU stub: scattered row/column-block subscriptions, and the LU
  app's three stage tasks per block step with pTaskInfo.taskId as the step.
* oracle/_ref/matrixMultiply_b200.exe: the reference's int matrixMultiply app
  with its own subtask_gpu_cuda kernel file (unchanged), one output row per
  subtask, on the runtime's CPU stub.
"""
from __future__ import annotations

import os
import subprocess

import pytest

from conftest import ROOT

SELFTEST = os.path.join(ROOT, "tests", "runtime", "_build", "rt_selftest")
APP = os.path.join(ROOT, "oracle", "_ref", "imageFiltering_b200.exe")
MM_APP = os.path.join(ROOT, "oracle", "_ref", "matrixMultiplyBlas_b200.exe")
LU_APP = os.path.join(ROOT, "oracle", "_ref", "luDecomposition_cpu.exe")
INT_MM_APP = os.path.join(ROOT, "oracle", "_ref", "matrixMultiply_b200.exe")


@pytest.fixture(scope="module")
def selftest():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "runtime")], check=True)
    return SELFTEST


def run(cmd, timeout=300, env=None):
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout,
                       env=None if env is None else dict(os.environ, **env))
    return p.returncode, p.stdout + p.stderr


@pytest.mark.parametrize("name", ["views_cpu", "views_cpu_compact", "errors", "timeout", "reduce_cpu",
                                  "redistribute_cpu"])
def test_runtime_cpu(selftest, name):
    rc, out = run([selftest, name])
    assert rc == 0 and f"PASS {name}" in out, out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["views_gpu", "views_gpu_compact", "chain", "write_through", "mix", "reduce_gpu",
                                  "sentinel_gpu", "redistribute_gpu"])
def test_runtime_gpu(selftest, name):
    rc, out = run([selftest, name])
    assert rc == 0 and f"PASS {name}" in out, out


def app_or_skip(path=APP):
    if not os.path.exists(path):
        pytest.skip("reference app not built (oracle/ref/Makefile needs the reference tree)")
    return path


def test_reference_app_cpu_mode_on_b200_runtime():
    """Parallel mode 1 (local CPU): subscriptions and views of the runtime
    drive the reference's own CPU callback across 3 chained tasks."""
    rc, out = run([app_or_skip(), "1", "1", "0", "2", "1", "4100", "2100", "3"])
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out


@pytest.mark.gpu
@pytest.mark.parametrize("args", [["2", "0", "4100", "2100", "3"], ["1", "1", "8192", "8192", "2"],
                                  ["3", "2", "777", "513", "2"]])
def test_reference_app_gpu_mode(args):
    """Parallel mode 2 (local GPU): the unchanged app runs its subtasks on the
    B200 stencil through the runtime (batched into one launch per task) and
    compares with its serial CPU run."""
    rc, out = run([app_or_skip(), "1", "2", "0"] + args, timeout=600)
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out


@pytest.mark.gpu
def test_reference_app_single_gpu_mode():
    """Run mode 4: the app's single-GPU path (singleGpuImageFilter) vs serial."""
    rc, out = run([app_or_skip(), "4", "2", "0", "2", "0", "3000", "1000", "1"])
    assert rc == 0 and "Single GPU Task's Sequential Comparison Test Passed" in out, out


@pytest.mark.parametrize("n", ["300", "1024", "4096"])
def test_reference_matrix_multiply_app_cpu_mode(n):
    """The unchanged matrixMultiplyBlas app, parallel mode 1: (n / min(n, 2048))^2
    subtasks (4 at 4096) over row-block / column-block / block subscriptions,
    compared by the app with its serial cblas_sgemm (relative 1e-5 per element)."""
    rc, out = run([app_or_skip(MM_APP), "1", "1", "0", n])
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out


def test_reference_lu_app_cpu_mode():
    """The unchanged luDecomposition app, parallel mode 1, 4096 = 2 x 2 blocks of
    2048: LU_DECOMPOSE, HORZ_VERT_COMP (2 subtasks), DIAGONAL_COMP, LU_DECOMPOSE as
    four tasks on one address space.  The app does not compare fp32 results
    (luDecomposition.cpp:593-595); tests/test_blas_ref_oracle.py checks the same
    stage sequence against the FP64 Crout factors."""
    rc, out = run([app_or_skip(LU_APP), "1", "1", "0", "4096"])
    assert rc == 0 and "Parallel Task 1 Execution Time" in out and "Failed" not in out, out


@pytest.mark.parametrize("n", ["1000", "257"])
def test_reference_int_matrix_multiply_app_cpu_mode(n):
    """The unchanged int matrixMultiply app, parallel mode 1: n subtasks of one
    output row each, every subtask subscribing the whole of B, compared by the
    app with its serial run."""
    rc, out = run([app_or_skip(INT_MM_APP), "1", "1", "0", n])
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out


@pytest.mark.gpu
@pytest.mark.parametrize("batch", ["grouped", "per_subtask"])
@pytest.mark.parametrize("n", ["1024", "4096"])
def test_reference_matrix_multiply_app_gpu_mode(n, batch):
    """The unchanged matrixMultiplyBlas app, parallel mode 2 (local GPU): its
    subtasks run on the tcgen05 BF16x3 GEMM of libpmb_app_matrixMultiplyBlas --
    through its batch hook (each half of a task's C blocks as one grouped
    product launch) or, with PMB_NO_BATCH=1, through matrixMultiply_cudaLaunchFunc
    per subtask -- and the app compares them with its serial cblas_sgemm at
    relative 1e-5 per element."""
    env = {"PMB_NO_BATCH": "1"} if batch == "per_subtask" else None
    rc, out = run([app_or_skip(MM_APP), "1", "2", "0", n], timeout=600, env=env)
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out


@pytest.mark.gpu
@pytest.mark.parametrize("n", ["1000", "257"])
def test_reference_int_matrix_multiply_app_gpu_mode(n):
    """The unchanged int matrixMultiply app, parallel mode 2: the runtime
    launches the app's own subtask_gpu_cuda kernel (matrixMultiplyCUDA.cu,
    compiled for sm_100a) per subtask and the app compares with its serial run."""
    rc, out = run([app_or_skip(INT_MM_APP), "1", "2", "0", n], timeout=600)
    assert rc == 0 and "Serial Comparison Test Passed" in out and "Failed" not in out, out
