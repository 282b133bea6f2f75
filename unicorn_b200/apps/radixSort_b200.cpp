// B200 GPU callback of the radixSort app's rounds (see radixSort_b200.h): the
// slice is copied to the output view and sorted there in one onesweep pass on
// the round's digit (pmb_radix_sort_u32, the alternate buffer and the sort's
// state in the subtask's reserved device memory); the pass's digit histogram
// is copied into the subtask's scratch buffer as the round's bin counts.
// The redistribution callback is the reference's, on the current API.
#include "radixSort_b200.h"

#include "pmb_capi.h"

namespace radixSort {

using namespace pm;

namespace {

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

size_t radixSortReservedBytes(size_t elems, int bitsPerRound) {
    return align256(elems * sizeof(uint32_t)) + pmb_radix_sort_scratch_bytes(elems, bitsPerRound);
}

pmStatus radixSort_cudaLaunchFunc(pmTaskInfo pTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream) {
    const radixSortTaskConf* conf = static_cast<const radixSortTaskConf*>(pTaskInfo.taskConf);
    const pmMemInfo& in = pSubtaskInfo.memInfo[0];
    const pmMemInfo& out = pSubtaskInfo.memInfo[1];
    const size_t n = in.length / sizeof(uint32_t);
    if (out.length < in.length || !pSubtaskInfo.gpuContext.scratchBuffer) return pmInvalidIndex;
    const int bits = conf->bitsPerRound;
    char* reserved = static_cast<char*>(pSubtaskInfo.gpuContext.reservedGlobalMem);
    uint32_t* alt = reinterpret_cast<uint32_t*>(reserved);
    void* state = reserved + align256(n * sizeof(uint32_t));
    const size_t state_bytes = pmb_radix_sort_scratch_bytes(n, bits);
    int st = pmb_memcpy_async(out.ptr, in.ptr, in.length, PMB_D2D, pCudaStream);
    if (st == PMB_SUCCESS)
        st = pmb_radix_sort_u32(static_cast<uint32_t*>(out.ptr), alt, n, conf->round * bits, (conf->round + 1) * bits,
                                bits, state, state_bytes, pCudaStream);
    if (st == PMB_SUCCESS)  // the pass's histogram: uint32 counts per digit
        st = pmb_radix_sort_histogram(state, bits, pSubtaskInfo.gpuContext.scratchBuffer, pCudaStream);
    return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st);
}

pmStatus radixSortDataRedistribution(pmTaskInfo pTaskInfo, pmDeviceInfo pDeviceInfo, pmSubtaskInfo pSubtaskInfo) {
    const radixSortTaskConf* conf = static_cast<const radixSortTaskConf*>(pTaskInfo.taskConf);
    const uint32_t* bins = static_cast<const uint32_t*>(pmGetScratchBuffer(
        pTaskInfo.taskHandle, pDeviceInfo.deviceHandle, pSubtaskInfo.subtaskId, pSubtaskInfo.splitInfo,
        SUBTASK_TO_POST_SUBTASK, 0, nullptr));
    if (!bins) return pmInvalidIndex;
    const int digits = 1 << conf->bitsPerRound;
    size_t offset = 0;
    for (int k = 0; k < digits; ++k) {
        const size_t bytes = static_cast<size_t>(bins[k]) * sizeof(uint32_t);
        const pmStatus st = pmRedistributeData(pTaskInfo.taskHandle, pDeviceInfo.deviceHandle, pSubtaskInfo.subtaskId,
                                               pSubtaskInfo.splitInfo, 1, offset, bytes,
                                               static_cast<uint>(pTaskInfo.subtaskCount * k + pSubtaskInfo.subtaskId));
        if (st != pmSuccess) return st;
        offset += bytes;
    }
    return pmSuccess;
}

}  // namespace radixSort
