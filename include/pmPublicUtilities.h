/*
 * pmPublicUtilities.h -- reduction helpers and file mapping of the pm:: API.
 * Same names, enumerator values and signatures as Unicorn's
 * source/code/inc/pmPublicUtilities.h (apps compile against them unchanged).
 */
#ifndef PM_PUBLIC_UTILITIES_H_B200
#define PM_PUBLIC_UTILITIES_H_B200
#define __PM_PUBLIC_UTILITIES__

#include "pmPublicDefinitions.h"

namespace pm
{
    typedef enum pmReductionOpType
    {
        REDUCE_ADD,
        REDUCE_MIN,
        REDUCE_MAX,
        REDUCE_PRODUCT,
        REDUCE_LOGICAL_AND,
        REDUCE_BITWISE_AND,
        REDUCE_LOGICAL_OR,
        REDUCE_BITWISE_OR,
        REDUCE_LOGICAL_XOR,
        REDUCE_BITWISE_XOR,
        MAX_REDUCTION_OP_TYPES
    } pmReductionOpType;

    typedef enum pmReductionDataType
    {
        REDUCE_INTS,
        REDUCE_UNSIGNED_INTS,
        REDUCE_LONGS,
        REDUCE_UNSIGNED_LONGS,
        REDUCE_FLOATS,
        REDUCE_DOUBLES,
        MAX_REDUCTION_DATA_TYPES
    } pmReductionDataType;

    /* Built-in element-wise reduction of two subtasks' write subscriptions. */
    pmDataReductionCallback pmGetSubtaskReductionCallbackImpl(pmReductionOpType pOperation, pmReductionDataType pDataType);

    /* Reduce subtask 2's output into subtask 1's (callable from a reduction callback). */
    pmStatus pmReduceSubtasks(pmTaskHandle pTaskHandle, pmDeviceHandle pDevice1Handle, unsigned long pSubtask1Id, pmSplitInfo& pSplitInfo1, pmDeviceHandle pDevice2Handle, unsigned long pSubtask2Id, pmSplitInfo& pSplitInfo2, pmReductionOpType pOperation, pmReductionDataType pDataType);

    const size_t MAX_FILE_SIZE_LEN = 2048;

    void* pmGetMappedFile(const char* pPath);
    pmStatus pmMapFile(const char* pPath);
    pmStatus pmUnmapFile(const char* pPath);
    pmStatus pmMapFiles(const char* const* pPaths, uint pFileCount);
    pmStatus pmUnmapFiles(const char* const* pPaths, uint pFileCount);
}

#endif
