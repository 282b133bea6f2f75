"""The drop-in boundary on the CPU: libpmlib.so exports every pm:: function
that include/pmPublicDefinitions.h and include/pmPublicUtilities.h declare,
under the exact C++ signature an unchanged app links against.

A translation unit that takes the address of each declared function through
a cast to its declared type (which selects the overload and so the mangled
name) is compiled against the headers and linked against libpmlib.so with
--no-undefined: a missing export or a signature drift fails the link."""
from __future__ import annotations

import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADERS = ["pmPublicDefinitions.h", "pmPublicUtilities.h"]
LIB = os.path.join(ROOT, "unicorn_b200", "libpmlib.so")

# A declaration on one line at namespace scope: return type, name, parameters.
DECL = re.compile(r"^    (?!inline\b|typedef\b|return\b)([A-Za-z_][\w\s\*&:]*?[\s\*&])(pm[A-Z]\w*)\s*\(([^;{]*)\)\s*;\s*$")


def declarations() -> list[tuple[str, str, str]]:
    out = []
    for h in HEADERS:
        with open(os.path.join(ROOT, "include", h)) as fh:
            for line in fh:
                m = DECL.match(line.rstrip("\n"))
                if m:
                    out.append((m.group(1).strip(), m.group(2), m.group(3).strip()))
    return out


def test_header_declarations_parsed():
    names = {n for _, n, _ in declarations()}
    # the API surface an app reaches (reference inc/pmPublicDefinitions.h, inc/pmPublicUtilities.h)
    expect = {"pmGetLibVersion", "pmGetLastError", "pmInitialize", "pmFinalize", "pmGetHostId", "pmGetHostCount",
              "pmRegisterCallbacks", "pmReleaseCallbacks", "pmCreateMemory", "pmCreateMemory2D", "pmReleaseMemory",
              "pmFetchMemory", "pmFetchMemoryRange", "pmGetRawMemPtr", "pmSubscribeToMemory", "pmRedistributeData",
              "pmSetCudaLaunchConf", "pmReserveCudaGlobalMem", "pmSubmitTask", "pmReleaseTask",
              "pmWaitForTaskCompletion", "pmGetTaskExecutionTimeInSecs", "pmReleaseTaskAndResources",
              "pmReleaseScratchBuffer", "pmGetLastReductionScratchBuffer", "pmGetRedistributionMetadata",
              "pmGetSubtaskReductionCallbackImpl", "pmReduceSubtasks", "pmGetMappedFile", "pmMapFile",
              "pmUnmapFile", "pmMapFiles", "pmUnmapFiles"}
    assert expect <= names, expect - names
    assert sum(1 for _, n, _ in declarations() if n == "pmSubscribeToMemory") == 2


def test_libpmlib_exports_every_declared_function(tmp_path):
    if not os.path.exists(LIB):
        pytest.skip("libpmlib.so not built")
    lines = ['#include "pmPublicDefinitions.h"', '#include "pmPublicUtilities.h"', "using namespace pm;",
             "int main(int argc, char**) {", "    void* volatile sink;"]
    for ret, name, params in declarations():
        lines.append(f"    sink = reinterpret_cast<void*>(static_cast<{ret} (*)({params})>(&pm::{name}));")
    # the inline pmGetScratchBuffer calls the library's pmGetScratchBufferHostFunc
    lines += ["    pmSplitInfo split;",
              "    if (argc > 1000) sink = pmGetScratchBuffer(nullptr, nullptr, 0, split, PRE_SUBTASK_TO_SUBTASK, 0, "
              "nullptr);"]
    lines += ["    (void)sink;", "    return 0;", "}"]
    src = tmp_path / "exports.cpp"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "exports"
    p = subprocess.run(["g++", "-std=c++11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", os.path.dirname(LIB), "-lpmlib", "-Wl,--no-undefined",
                        "-Wl,--unresolved-symbols=ignore-in-shared-libs"], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-4000:]
