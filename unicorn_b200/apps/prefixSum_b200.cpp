// B200 GPU callbacks of the prefixSum app's two tasks (see prefixSum_b200.h):
// the slice scan runs pmb_inclusive_scan_u32_u64 (single-pass decoupled
// look-back) with its state in the subtask's reserved device memory, and the
// add of the preceding slices' total runs pmb_add_u64_scalar.  Both only
// enqueue work on the subtask's stream.
#include "prefixSum_b200.h"

#include "pmb_capi.h"

namespace prefixSum {

using namespace pm;

size_t prefixSumReservedBytes(size_t elems) { return pmb_scan_scratch_bytes(elems); }

pmStatus prefixSum_cudaLaunchFunc(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream) {
    const pmMemInfo& in = pSubtaskInfo.memInfo[0];
    const pmMemInfo& out = pSubtaskInfo.memInfo[1];
    const size_t n = in.length / sizeof(uint32_t);
    if (out.length < n * sizeof(uint64_t)) return pmInvalidIndex;
    const int st = pmb_inclusive_scan_u32_u64(static_cast<const uint32_t*>(in.ptr), static_cast<uint64_t*>(out.ptr), n,
                                              pSubtaskInfo.gpuContext.reservedGlobalMem, prefixSumReservedBytes(n),
                                              pCudaStream);
    return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st);
}

pmStatus elemAdd_cudaLaunchFunc(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream) {
    const pmMemInfo& total = pSubtaskInfo.memInfo[0];
    const pmMemInfo& out = pSubtaskInfo.memInfo[1];
    const int st = pmb_add_u64_scalar(static_cast<uint64_t*>(out.ptr), out.length / sizeof(uint64_t),
                                      static_cast<const uint64_t*>(total.ptr), pCudaStream);
    return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st);
}

}  // namespace prefixSum
