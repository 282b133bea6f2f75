// prefixSum app interface shared with the B200 GPU callbacks.
//
// The reference app (testSuite/prefixSum/source/code/src/prefixSum.cpp,
// prefixSum.h) is written against an older pm:: API (pSubtaskInfo.inputMem /
// outputMem, 5-argument CREATE_TASK) and does not compile against the current
// one; these callbacks keep its two-task flow and callback names on the
// current API: task 1 scans every subtask's slice (prefixSum_cudaLaunchFunc,
// prefixSumCUDA.cu:262-267), the app scans the slice totals on the host
// (PopulateAuxMem, prefixSum.cpp:191-214), task 2 adds total i to slice i + 1
// (elemAdd, prefixSum.cpp:100-131 and prefixSumCUDA.cu:143-158).  Widened
// to uint32 input and uint64 sums: memInfo[0] is the uint32 input slice,
// memInfo[1] the uint64 output slice (task 1); memInfo[0] the uint64 total,
// memInfo[1] the uint64 output slice (task 2).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "pmPublicDefinitions.h"

namespace prefixSum {

typedef struct prefixSumTaskConf {
    uint64_t arrayLen;
    uint64_t elemsPerSubtask;
} prefixSumTaskConf;

// Device memory a task-1 subtask of `elems` elements must reserve
// (pmReserveCudaGlobalMem) for the scan's look-back state.
size_t prefixSumReservedBytes(size_t elems);

pm::pmStatus prefixSum_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                      pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
pm::pmStatus elemAdd_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                    pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);

}  // namespace prefixSum
