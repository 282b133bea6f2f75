// matrixMultiplyBlas app interface shared with the B200 GPU callbacks.
//
// Names, signatures and the task-configuration layout are those of
// testSuite/matrixMultiplyBlas/source/code/inc/matrixMultiplyBlas.h (:36-89,
// float build): the app passes matrixMultiplyTaskConf through taskConf.
// GetSplitData is defined by the app (matrixMultiplyBlas.cpp:67-88).
#pragma once

#include <stddef.h>

#include "pmPublicDefinitions.h"

namespace matrixMultiplyBlas {

enum memIndexB200 { kMatrixA = 0, kMatrixB = 1, kMatrixC = 2 };

typedef struct matrixMultiplyTaskConf {
    size_t matrixDim;
    size_t blockDim;
} matrixMultiplyTaskConf;

// Defined by the app.
bool GetSplitData(size_t* pBlockOffset, size_t* pBlockHeight, matrixMultiplyTaskConf* pTaskConf,
                  pm::pmSplitInfo& pSplitInfo);

// Provided by the B200 library in place of matrixMultiplyBlasCUDA.cu.
pm::pmStatus matrixMultiply_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                           pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
int singleGpuMatrixMultiply(float* pInputMatrices, float* pOutputMatrix, int pDim);

}  // namespace matrixMultiplyBlas
