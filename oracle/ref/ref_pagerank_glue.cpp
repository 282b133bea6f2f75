/*
 * ref_pagerank_glue.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own pageRank_cpu (testSuite/pageRank/source/code/src/
 * pageRank.cpp:336-378, compiled unchanged from the reference tree by
 * oracle/ref/Makefile) on a graph handed over as out-adjacency lists.  The
 * graph is laid out in the reference's web-dump page format (per page: the
 * out-link count, then maxOutlinks 1-based target ids, pageRank.cpp:53-111)
 * in one in-memory "file" that pmGetMappedFile returns; one subtask covers
 * every page and each iteration is one call, the previous ranks passed as the
 * input address space (pageRankDataDistribution, :278-307).
 */
#include <cstdint>
#include <cstring>
#include <vector>

#include "commonAPI.h"
#include "pageRank.h"

namespace {
std::vector<unsigned int> g_dump;
}

namespace pm {
void* pmGetMappedFile(const char*) { return g_dump.data(); }
pmStatus pmMapFiles(const char* const*, uint) { return pmSuccess; }
pmStatus pmUnmapFiles(const char* const*, uint) { return pmSuccess; }
uint pmGetHostCount() { return 1; }
pmStatus pmSubscribeToMemory(pmTaskHandle, pmDeviceHandle, ulong, pmSplitInfo&, uint, pmSubscriptionType,
                             const pmSubscriptionInfo&) { return pmSuccess; }
pmStatus pmSubmitTask(pmTaskDetails, pmTaskHandle*) { return pmStatusUnavailable; }
pmStatus pmFetchMemory(pmMemHandle) { return pmStatusUnavailable; }
pmStatus pmReleaseTask(pmTaskHandle) { return pmStatusUnavailable; }
pmStatus pmCreateMemory(size_t, pmMemHandle*) { return pmStatusUnavailable; }
pmStatus pmGetRawMemPtr(pmMemHandle, pmRawMemPtr*) { return pmStatusUnavailable; }
pmStatus pmReleaseMemory(pmMemHandle) { return pmStatusUnavailable; }
pmStatus pmWaitForTaskCompletion(pmTaskHandle) { return pmStatusUnavailable; }
pmDataReductionCallback pmGetSubtaskReductionCallbackImpl(pmReductionOpType, pmReductionDataType) { return NULL; }
}  // namespace pm

void commonStart(int, char**, initFunc, serialProcessFunc, singleGpuProcessFunc, parallelProcessFunc,
                 compareFunc, destroyFunc, callbackStruct*, size_t) {}
void commonFinish() {}
uint getAffinityCriterion() { return 0; }
double getCurrentTimeInSecs() { return 0.0; }
bool isMultiAssignEnabled() { return false; }
bool isComputeCommunicationOverlapEnabled() { return false; }

namespace pageRank {
pmStatus pageRank_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
}

extern "C" {

/* out_ptr[N+1] / out_dst[E]: out-adjacency (0-based targets, in the order the
 * reference would read them).  Runs `iters` iterations from the uniform
 * initial rank `init`; writes the final fp32 ranks to `out`.  Returns 0 on
 * success. */
int ref_pagerank(const uint32_t* out_ptr, const uint32_t* out_dst, uint32_t n, int iters, float init, float* out) {
    using namespace pageRank;
    uint32_t max_out = 0;
    for (uint32_t u = 0; u < n; ++u) max_out = out_ptr[u + 1] - out_ptr[u] > max_out ? out_ptr[u + 1] - out_ptr[u] : max_out;
    g_dump.assign(static_cast<size_t>(n) * (max_out + 1), 0u);
    for (uint32_t u = 0; u < n; ++u) {
        unsigned int* page = &g_dump[static_cast<size_t>(u) * (max_out + 1)];
        page[0] = out_ptr[u + 1] - out_ptr[u];
        for (uint32_t k = out_ptr[u]; k < out_ptr[u + 1]; ++k) page[1 + k - out_ptr[u]] = out_dst[k] + 1;
    }
    pageRankTaskConf conf;
    std::memset(&conf, 0, sizeof(conf));
    conf.totalWebPages = n;
    conf.maxOutlinksPerWebPage = max_out;
    conf.webPagesPerFile = n;
    conf.webPagesPerSubtask = n;
    conf.initialPageRank = init;
    std::vector<float> prev(n, init), cur(n, 0.0f);
    for (int it = 0; it < iters; ++it) {
        conf.iteration = static_cast<unsigned int>(it);
        pmTaskInfo ti;
        ti.taskConf = &conf;
        ti.taskConfLength = sizeof(conf);
        ti.subtaskCount = 1;
        pmDeviceInfo di;
        di.deviceType = pm::CPU;
        pmSubtaskInfo si;
        si.subtaskId = 0;
        si.memCount = MAX_MEM_INDICES;
        si.memInfo[OUTPUT_MEM_INDEX] = pmMemInfo(cur.data(), NULL, cur.data(), sizeof(float) * n, SUBSCRIPTION_NATURAL);
        si.memInfo[INPUT_MEM_INDEX] = pmMemInfo(prev.data(), prev.data(), NULL, sizeof(float) * n, SUBSCRIPTION_NATURAL);
        if (pageRank_cpu(ti, di, si) != pmSuccess) return 1;
        prev.swap(cur);
    }
    std::memcpy(out, prev.data(), sizeof(float) * n);
    return 0;
}

}  // extern "C"
