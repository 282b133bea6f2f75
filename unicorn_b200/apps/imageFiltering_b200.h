// imageFiltering app interface shared with the B200 GPU callbacks.
//
// The names, signatures and the task-configuration layout below are those of
// testSuite/imageFiltering/source/code/inc/imageFiltering.h (:55-111, with
// LOAD_IMAGE_INTO_ADDRESS_SPACE and without USE_VARIABLE_SIZED_SUBTASKS, its
// defaults): the app passes imageFilterTaskConf through pmTaskDetails::taskConf
// and these callbacks read it, so the struct must keep this exact layout.
// GetSubtaskSubscription is defined by the app (imageFiltering.cpp:279-340);
// the callbacks call it, exactly as the reference's imageFilteringCUDA.cu does.
#pragma once

#include <stddef.h>

#include "pmPublicDefinitions.h"

namespace imageFiltering {

constexpr size_t kPixelCount = 3;       // PIXEL_COUNT
constexpr int kMaxFilterDim = 32;       // MAX_FILTER_DIM
constexpr int kMaxImagePathLength = 256;  // MAX_IMAGE_PATH_LENGTH

enum memIndexB200 { kInputMemIndex = 0, kOutputMemIndex = 1 };

typedef struct imageFilterTaskConf {
    size_t imageWidth;
    size_t imageHeight;
    size_t imageOffset;
    size_t imageBytesPerLine;
    size_t filterRadius;
    char imagePath[kMaxImagePathLength];
    char filter[kMaxFilterDim][kMaxFilterDim];
} imageFilterTaskConf;

// Defined by the app.
bool GetSubtaskSubscription(imageFilterTaskConf* pTaskConf, unsigned long pSubtaskId, pm::pmSplitInfo& pSplitInfo,
                            int* pStartCol, int* pEndCol, int* pStartRow, int* pEndRow);

// Provided by the B200 library in place of imageFilteringCUDA.cu.
size_t computeSubtaskReservedMemRequirement(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                            unsigned long pSubtaskId, int pSubscriptionStartCol,
                                            int pSubscriptionEndCol, int pSubscriptionStartRow,
                                            int pSubscriptionEndRow);
pm::pmStatus imageFilter_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                        pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
int singleGpuImageFilter(void* pInvertedImageData, size_t pImageWidth, size_t pImageHeight,
                         char pFilter[kMaxFilterDim][kMaxFilterDim], size_t pFilterRadius, size_t pImageBytesPerLine,
                         void* pOutputMem);

}  // namespace imageFiltering
