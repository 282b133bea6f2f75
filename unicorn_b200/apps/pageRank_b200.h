// pageRank app interface shared with the B200 GPU callbacks.
//
// The names, signatures and the task-configuration layout below are those of
// testSuite/pageRank/source/code/inc/pageRank.h (:34-79, PAGE_RANK_DATA_TYPE
// float, its default): the app passes pageRankTaskConf through
// pmTaskDetails::taskConf and these callbacks read it, so the struct must keep
// this exact layout.  LoadMappedFiles is defined by the app
// (pageRank.cpp:309-334); the GPU callback calls it, as the reference's
// pageRankCUDA.cu does.
#pragma once

#include "pmPublicDefinitions.h"

namespace pageRank {

constexpr int kPageRankIterations = 2;       // PAGE_RANK_ITERATIONS
constexpr float kDampeningFactor = 0.85f;    // DAMPENING_FACTOR
constexpr int kMaxBasePathLength = 256;      // MAX_BASE_PATH_LENGTH

enum memIndexB200 { kOutputMemIndex = 0, kInputMemIndex = 1 };

typedef struct pageRankTaskConf {
    unsigned int totalWebPages;
    unsigned int maxOutlinksPerWebPage;
    unsigned int webPagesPerFile;
    unsigned int webPagesPerSubtask;
    unsigned int iteration;
    float initialPageRank;
    char basePath[kMaxBasePathLength];
} pageRankTaskConf;

// Defined by the app: the mapped page files of one subtask (new[]'d array).
void** LoadMappedFiles(pageRankTaskConf* pTaskConf, unsigned long pSubtaskId);

// Provided by the B200 library in place of pageRankCUDA.cu.
pm::pmStatus pageRank_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                     pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
int singleGpuPageRank(pageRankTaskConf& pTaskConf, unsigned int* pWebDump, void* pOutputMem);

}  // namespace pageRank
