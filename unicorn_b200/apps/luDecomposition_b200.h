// luDecomposition app interface shared with the B200 GPU callbacks.
//
// Names, signatures, BLOCK_DIM and the task-configuration layout are those of
// testSuite/luDecomposition/source/code/inc/luDecomposition.h (:36-38, :64-110,
// float build): the app's three stage tasks (LU_DECOMPOSE, HORZ_VERT_COMP,
// DIAGONAL_COMP) pass luTaskConf through taskConf and subscribe BLOCK_DIM x
// BLOCK_DIM column-major blocks of one address space; the callbacks locate the
// blocks from the subscription views exactly as the reference's
// luDecompositionCUDA.cu does, so BLOCK_DIM must equal the app's.
#pragma once

#include <stddef.h>

#include "pmPublicDefinitions.h"

namespace luDecomposition {

constexpr size_t kBlockDim = 2048;  // BLOCK_DIM
constexpr unsigned kOutputMemIndex = 0;

// BLOCK_OFFSET_IN_ELEMS: element offset of block (blockRow, blockCol).
constexpr size_t block_offset(size_t row, size_t col, size_t dim) { return (row + col * dim) * kBlockDim; }

typedef struct luTaskConf {
    size_t matrixDim;
} luTaskConf;

// Provided by the B200 library in place of luDecompositionCUDA.cu.
pm::pmStatus luDecomposition_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                            pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
pm::pmStatus horizVertComp_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                          pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
pm::pmStatus diagComp_cudaLaunchFunc(pm::pmTaskInfo pTaskInfo, pm::pmDeviceInfo pDeviceInfo,
                                     pm::pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
int singleGpuLUDecomposition(float* pMatrix, size_t pDim);

}  // namespace luDecomposition
