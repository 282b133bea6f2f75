// radixSort app interface shared with the B200 GPU callbacks.
//
// The reference app (testSuite/radixSort/source/code/src/radixSort.cpp,
// radixSort.h) is written against an older pm:: API and does not compile
// against the current one; these callbacks keep its per-round structure on the
// current API: every subtask sorts its slice stably on the round's digit and
// leaves the digit counts in its SUBTASK_TO_POST_SUBTASK scratch buffer
// (radixSort_cpu, radixSort.cpp:127-134), and the redistribution callback
// names each digit's keys with order subtaskCount * digit + subtaskId
// (radixSortDataRedistribution, :136-148), so the rebuilt address space is
// the keys stably ordered by that digit.  memInfo[0] is the input slice,
// memInfo[1] the output slice (uint32 keys).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "pmPublicDefinitions.h"

namespace radixSort {

typedef struct radixSortTaskConf {
    uint64_t arrayLen;
    uint64_t elemsPerSubtask;
    int round;         // LSD round: digit bits [round * bits, (round + 1) * bits)
    int bitsPerRound;  // 4 (the reference's BITS_PER_ROUND) or 8
} radixSortTaskConf;

// Device memory a subtask sorting `elems` keys must reserve
// (pmReserveCudaGlobalMem): the second key buffer and the sort's state.
size_t radixSortReservedBytes(size_t elems, int bitsPerRound);

pm::pmStatus radixSort_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                      pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
pm::pmStatus radixSortDataRedistribution(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                         pm::pmSubtaskInfo pSubtaskInfo);

}  // namespace radixSort
