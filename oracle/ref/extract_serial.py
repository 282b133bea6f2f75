"""Build step for the test checkers (TEST INFRASTRUCTURE ONLY).

The reference's prefixSum.cpp and radixSort.cpp do not compile as whole files
(their task code uses an older pm:: API: pSubtaskInfo.inputMem, 5-argument
pmSubscribeToMemory and CREATE_TASK), but their serial CPU functions are plain
C++.  This script cuts those functions, unchanged, out of the reference files
and writes one translation unit with C entry points around them:

* prefixSum.cpp: serialPrefixSum (:47-53);
* radixSort.cpp: the BIT_MASK / *_RIGHT_SHIFT_BITS macros (:46-49),
  serialRadixSortRound, serialMsbRadixSortRound, serialLsbRadixSortRound and
  serialLsbRadixSort (:51-114).

With --reducer it instead cuts the subtask-reduction fold out of the
reference runtime's source/code/src/pmReducer.cpp: getBitwiseOperatableType
(:408-424) and the member template pmReducer::ReduceMemories (:590-700), which
compiles unchanged against a stand-in declaration of the class (the rest of
pmReducer needs the whole runtime and MPI); C entry points dispatch on the
data type as pmReducer::ReduceExternalMemory does (:502-540).

The output goes to oracle/_ref/ (git-ignored) and is compiled by
oracle/ref/Makefile with the reference's own headers (prefixSum.h,
radixSort.h).  A missing function fails the build.

Usage: python extract_serial.py <reference testSuite dir> <output .cpp>
       python extract_serial.py --reducer <reference pmReducer.cpp> <output .cpp>
"""
from __future__ import annotations

import os
import sys


def function(lines: list[str], signature: str) -> list[str]:
    """The lines of the function whose definition starts with `signature`,
    through the closing brace in column 0."""
    for i, line in enumerate(lines):
        if line.startswith(signature):
            for j in range(i + 1, len(lines)):
                if lines[j].rstrip() == "}":
                    return lines[i:j + 1]
    raise SystemExit(f"extract_serial: '{signature}' not found")


def macro(lines: list[str], name: str) -> str:
    for line in lines:
        if line.startswith(f"#define {name}"):
            return line
    raise SystemExit(f"extract_serial: macro {name} not found")


def reducer(src: str, out: str) -> None:
    with open(src) as fh:
        rd = fh.read().splitlines()
    start = next(i for i, line in enumerate(rd) if line.startswith("struct getBitwiseOperatableType"))
    bitwise = rd[start - 1:]  # the template<> line before the primary template
    end = next(i for i, line in enumerate(bitwise) if line.startswith("    typedef ulong type;"))
    bitwise = bitwise[:end + 2]
    fold = function(rd, "void pmReducer::ReduceMemories(")
    text = [
        "// Generated by oracle/ref/extract_serial.py from the reference's pmReducer.cpp",
        "// (getBitwiseOperatableType and pmReducer::ReduceMemories, unchanged).  Test infrastructure only.",
        "#include <algorithm>",
        "#include <cstddef>",
        '#include "pmPublicDefinitions.h"',
        '#include "pmPublicUtilities.h"',
        "namespace pm {",
        "struct pmFatalErrorException {};",
        "#define PMTHROW(x) throw x",
        "class pmReducer {",
        "  public:",
        "    template<typename datatype>",
        "    static void ReduceMemories(datatype* pShadowMem1, datatype* pShadowMem2, size_t pDataCount,",
        "                               pmReductionOpType pReductionType);",
        "};",
        *bitwise,
        "template<typename datatype>",
        *fold,
        "}  // namespace pm",
        'extern "C" int ref_reduce_memories(int op, int type, void* a, void* b, size_t count) {',
        "    using namespace pm;",
        "    const pmReductionOpType o = static_cast<pmReductionOpType>(op);",
        "    try {",
        "        switch (type) {",
        "            case REDUCE_INTS: pmReducer::ReduceMemories<int>((int*)a, (int*)b, count, o); break;",
        "            case REDUCE_UNSIGNED_INTS: pmReducer::ReduceMemories<uint>((uint*)a, (uint*)b, count, o); break;",
        "            case REDUCE_LONGS: pmReducer::ReduceMemories<long>((long*)a, (long*)b, count, o); break;",
        "            case REDUCE_UNSIGNED_LONGS: pmReducer::ReduceMemories<ulong>((ulong*)a, (ulong*)b, count, o); break;",
        "            case REDUCE_FLOATS: pmReducer::ReduceMemories<float>((float*)a, (float*)b, count, o); break;",
        "            case REDUCE_DOUBLES: pmReducer::ReduceMemories<double>((double*)a, (double*)b, count, o); break;",
        "            default: return 1;",
        "        }",
        "    } catch (...) {",
        "        return 2;",
        "    }",
        "    return 0;",
        "}",
    ]
    with open(out, "w") as fh:
        fh.write("\n".join(text) + "\n")


def main() -> None:
    if sys.argv[1] == "--reducer":
        reducer(sys.argv[2], sys.argv[3])
        return
    ts, out = sys.argv[1], sys.argv[2]
    with open(os.path.join(ts, "prefixSum", "source", "code", "src", "prefixSum.cpp")) as fh:
        ps = fh.read().splitlines()
    with open(os.path.join(ts, "radixSort", "source", "code", "src", "radixSort.cpp")) as fh:
        rs = fh.read().splitlines()
    text = [
        "// Generated by oracle/ref/extract_serial.py from the reference's prefixSum.cpp and",
        "// radixSort.cpp (serial CPU functions, unchanged).  Test infrastructure only.",
        "#include <string.h>",
        '#include "pmPublicDefinitions.h"',
        "using namespace pm;",
        '#include "prefixSum.h"',
        '#include "radixSort.h"',
        "namespace prefixSum {",
        *function(ps, "void serialPrefixSum("),
        "}  // namespace prefixSum",
        "namespace radixSort {",
        *(macro(rs, m) for m in ("BIT_MASK", "LSB_RIGHT_SHIFT_BITS", "MSB_RIGHT_SHIFT_BITS", "RIGHT_SHIFT_BITS")),
        *function(rs, "void serialRadixSortRound("),
        *function(rs, "void serialMsbRadixSortRound("),
        *function(rs, "void serialLsbRadixSortRound("),
        *function(rs, "void serialLsbRadixSort("),
        "}  // namespace radixSort",
        'extern "C" {',
        "int ref_radix_bits_per_round(void) { return radixSort::BITS_PER_ROUND; }",
        "int ref_radix_total_rounds(void) { return radixSort::TOTAL_ROUNDS; }",
        "void ref_serial_prefix_sum_i32(int* in, int* out, unsigned n) { prefixSum::serialPrefixSum(in, out, n); }",
        "void ref_serial_lsb_radix_round_u32(unsigned* in, unsigned* out, unsigned n, int round, int* bins) {",
        "    radixSort::serialLsbRadixSortRound(in, out, n, round, bins);",
        "}",
        "void ref_serial_lsb_radix_sort_u32(unsigned* in, unsigned* out, unsigned n, int rounds) {",
        "    radixSort::serialLsbRadixSort(in, out, n, rounds);",
        "}",
        "}",
    ]
    with open(out, "w") as fh:
        fh.write("\n".join(text) + "\n")


if __name__ == "__main__":
    main()
