/*
 * ref_blas_stubs.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Shared by the glue files that drive the reference's BLAS apps' CPU
 * callbacks outside the reference runtime (ref_mm_glue.cpp,
 * ref_lu_glue.cpp): a recorder for the pmSubscribeToMemory calls a data
 * distribution callback makes, NATURAL views built from it (address-space
 * base + the lowest subscribed offset of each memory index, which is where
 * the reference runtime's natural view of a subtask starts), and stubs of
 * the commonAPI / pm:: functions the app files reference but the callbacks
 * never reach.  Include it once, after commonAPI.h and the app header.
 */
#pragma once

#include <cstddef>
#include <cstring>
#include <vector>

namespace refglue {
struct Sub {
    unsigned mem;
    pm::pmSubscriptionType type;
    pm::pmScatteredSubscriptionInfo info;
};
thread_local std::vector<Sub> t_subs;

// Lowest subscribed offset of memory index `mem`, or SIZE_MAX if none.
inline size_t lowest(unsigned mem) {
    size_t lo = (size_t)-1;
    for (const Sub& s : t_subs)
        if (s.mem == mem && s.info.offset < lo) lo = s.info.offset;
    return lo;
}
}  // namespace refglue

namespace pm {
pmStatus pmSubscribeToMemory(pmTaskHandle, pmDeviceHandle, ulong, pmSplitInfo&, uint pMemIndex,
                             pmSubscriptionType pType, const pmScatteredSubscriptionInfo& pInfo) {
    if (pMemIndex >= MAX_MEM_SECTIONS_PER_TASK) return pmInvalidIndex;
    refglue::t_subs.push_back({pMemIndex, pType, pInfo});
    return pmSuccess;
}
pmStatus pmSubmitTask(pmTaskDetails, pmTaskHandle*) { return pmStatusUnavailable; }
pmStatus pmFetchMemory(pmMemHandle) { return pmStatusUnavailable; }
pmStatus pmReleaseTask(pmTaskHandle) { return pmStatusUnavailable; }
pmStatus pmGetRawMemPtr(pmMemHandle, pmRawMemPtr*) { return pmStatusUnavailable; }
pmStatus pmReleaseMemory(pmMemHandle) { return pmStatusUnavailable; }
pmStatus pmCreateMemory2D(size_t, size_t, pmMemHandle*) { return pmStatusUnavailable; }
pmStatus pmWaitForTaskCompletion(pmTaskHandle) { return pmStatusUnavailable; }
pmStatus pmReleaseTaskAndResources(pmTaskDetails, pmTaskHandle) { return pmStatusUnavailable; }
}  // namespace pm

void commonStart(int, char**, initFunc, serialProcessFunc, singleGpuProcessFunc, parallelProcessFunc,
                 compareFunc, destroyFunc, callbackStruct*, size_t) {}
void commonFinish() {}
void DistributeMemory(pmMemHandle, memDistributionType, unsigned int, unsigned int, unsigned int,
                      unsigned int, bool) {}
uint getAffinityCriterion() { return 0; }
double getCurrentTimeInSecs() { return 0.0; }
bool isMultiAssignEnabled() { return false; }
bool isComputeCommunicationOverlapEnabled() { return false; }
bool isLazyMemEnabled() { return false; }
bool isCudaCacheEnabled() { return true; }
