/*
 * pmPublicDefinitions.h -- public C++ API of the B200 pmlib runtime (libpmlib.so).
 *
 * This header is a from-scratch restatement of the pm:: interface of Unicorn's
 * source/code/inc/pmPublicDefinitions.h.  Names, signatures, enumerator values
 * and struct member order are kept identical on purpose, because existing apps
 * are compiled against them and pass pmTaskInfo / pmSubtaskInfo BY VALUE into
 * CUDA kernels: the byte layout of those structs is part of the drop-in
 * contract.  Struct constructors are defined inline here (same default values
 * as the reference), so apps need no constructor symbols from the library.
 *
 * Differences in this runtime (one process, one CUDA device):
 *  - pmGetHostId() is always 0 and pmGetHostCount() always 1;
 *  - GPU_CUDA is always present in pmDeviceType and pmTaskDetails always
 *    carries cudaCacheEnabled (the reference gates both on SUPPORT_CUDA; every
 *    CUDA-enabled app build defines it);
 *  - scheduling policy, affinity and multi-assign fields are accepted and
 *    ignored (a single device executes every subtask).
 */
#ifndef PM_PUBLIC_DEFINITIONS_H_B200
#define PM_PUBLIC_DEFINITIONS_H_B200
#define __PM_PUBLIC_DEFINITIONS__

#include <stdlib.h>
#include <limits.h>

#ifndef SUPPORT_CUDA
#define SUPPORT_CUDA
#endif

namespace pm
{
    typedef unsigned short int ushort;
    typedef unsigned int uint;
    typedef unsigned long ulong;

    const size_t MAX_NAME_STR_LEN = 256;
    const size_t MAX_DESC_STR_LEN = 1024;
    const size_t MAX_CB_KEY_LEN = 128;
    const size_t MAX_MEM_SECTIONS_PER_TASK = 3;

    /* Outcome of every API call. */
    typedef enum pmStatus
    {
        pmSuccess = 0,
        pmOk,
        pmStatusUnavailable,
        pmFatalError,
        pmInitializationFailure,
        pmNetworkInitError,
        pmNetworkTerminationError,
        pmInvalidIndex,
        pmInvalidCommand,
        pmThreadingLibraryFailure,
        pmTimerFailure,
        pmMemoryError,
        pmNetworkError,
        pmIgnorableError,
        pmGraphicsCardError,
        pmBeyondComputationalLimits,
        pmUnrecognizedMemory,
        pmInvalidKey,
        pmMaxKeyLengthExceeded,
        pmDataProcessingFailure,
        pmNoCompatibleDevice,
        pmConfFileNotFound,
        pmInvalidOffset,
        pmInvalidCallbacks,
        pmUserError,
        pmMaxStatusValues
    } pmStatus;

    const char* pmGetLibVersion();
    const char* pmGetLastError();
    pmStatus pmInitialize();
    pmStatus pmFinalize();
    uint pmGetHostId();
    uint pmGetHostCount();

    typedef void* pmMemHandle;
    typedef void* pmRawMemPtr;
    typedef void* pmTaskHandle;
    typedef void* pmDeviceHandle;
    typedef void* pmCallbackHandle;
    typedef void* pmClusterHandle;

    typedef enum pmMemType
    {
        READ_ONLY,
        WRITE_ONLY,
        READ_WRITE,
        READ_ONLY_LAZY,
        WRITE_ONLY_LAZY,
        READ_WRITE_LAZY,
        MAX_MEM_TYPE
    } pmMemType;

    typedef enum pmSubscriptionType
    {
        READ_SUBSCRIPTION,
        WRITE_SUBSCRIPTION,
        READ_WRITE_SUBSCRIPTION
    } pmSubscriptionType;

    /* NATURAL: a subtask sees subscribed bytes at their address-space offsets.
     * COMPACT: subscribed pieces are packed back to back.
     * OPTIMAL: the runtime picks (COMPACT on the GPU, NATURAL on the CPU). */
    typedef enum pmSubscriptionVisibilityType
    {
        SUBSCRIPTION_NATURAL,
        SUBSCRIPTION_COMPACT,
        SUBSCRIPTION_OPTIMAL,
        MAX_SUBSCRIPTION_VISBILITY_TYPE
    } pmSubscriptionVisibilityType;

    /* A contiguous byte range of an address space. */
    typedef struct pmSubscriptionInfo
    {
        size_t offset;
        size_t length;

        pmSubscriptionInfo() : offset(0), length(0) {}
        pmSubscriptionInfo(size_t pOffset, size_t pLength) : offset(pOffset), length(pLength) {}
    } pmSubscriptionInfo;

    /* `count` ranges of `size` bytes, `step` bytes apart, the first at `offset`. */
    typedef struct pmScatteredSubscriptionInfo
    {
        size_t offset;
        size_t size;
        size_t step;
        size_t count;

        pmScatteredSubscriptionInfo() : offset(0), size(0), step(0), count(0) {}
        pmScatteredSubscriptionInfo(size_t pOffset, size_t pSize, size_t pStep, size_t pCount)
            : offset(pOffset), size(pSize), step(pStep), count(pCount) {}
    } pmScatteredSubscriptionInfo;

    /* Device-side buffers handed to a GPU subtask. */
    typedef struct pmGpuContext
    {
        void* scratchBuffer;
        void* reservedGlobalMem;

        pmGpuContext() : scratchBuffer(NULL), reservedGlobalMem(NULL) {}
    } pmGpuContext;

    typedef struct pmSplitInfo
    {
        uint splitId;
        uint splitCount;

        pmSplitInfo() : splitId(0), splitCount(0) {}
        pmSplitInfo(uint pSplitId, uint pSplitCount) : splitId(pSplitId), splitCount(pSplitCount) {}
    } pmSplitInfo;

    /* What one address space looks like to one subtask. */
    typedef struct pmMemInfo
    {
        pmRawMemPtr ptr;
        pmRawMemPtr readPtr;
        pmRawMemPtr writePtr;
        size_t length;
        pmSubscriptionVisibilityType visibilityType;

        pmMemInfo() : ptr(NULL), readPtr(NULL), writePtr(NULL), length(0), visibilityType(SUBSCRIPTION_NATURAL) {}
        pmMemInfo(pmRawMemPtr pPtr, pmRawMemPtr pReadPtr, pmRawMemPtr pWritePtr, size_t pLength)
            : ptr(pPtr), readPtr(pReadPtr), writePtr(pWritePtr), length(pLength), visibilityType(SUBSCRIPTION_NATURAL) {}
        pmMemInfo(pmRawMemPtr pPtr, pmRawMemPtr pReadPtr, pmRawMemPtr pWritePtr, size_t pLength, pmSubscriptionVisibilityType pVisibilityType)
            : ptr(pPtr), readPtr(pReadPtr), writePtr(pWritePtr), length(pLength), visibilityType(pVisibilityType) {}
    } pmMemInfo;

    typedef struct pmSubtaskInfo
    {
        ulong subtaskId;
        pmMemInfo memInfo[MAX_MEM_SECTIONS_PER_TASK];
        uint memCount;
        pmGpuContext gpuContext;
        pmSplitInfo splitInfo;

        pmSubtaskInfo() : subtaskId(ULONG_MAX), memCount(0) {}
        pmSubtaskInfo(ulong pSubtaskId, pmMemInfo* pMemInfo, uint pMemCount) : subtaskId(pSubtaskId), memCount(pMemCount)
        {
            for(uint i = 0; i < pMemCount && i < MAX_MEM_SECTIONS_PER_TASK; ++i)
                memInfo[i] = pMemInfo[i];
        }
    } pmSubtaskInfo;

    typedef struct pmTaskInfo
    {
        pmTaskHandle taskHandle;
        void* taskConf;
        uint taskConfLength;
        ulong taskId;
        ulong subtaskCount;
        ushort priority;
        uint originatingHost;

        pmTaskInfo() : taskHandle(NULL), taskConf(NULL), taskConfLength(0), taskId(0), subtaskCount(0), priority(0), originatingHost(0) {}
    } pmTaskInfo;

    typedef struct pmDataTransferInfo
    {
        pmMemHandle memHandle;
        size_t memLength;
        size_t* operatedMemLength;
        pmMemType memType;
        uint srcHost;
        uint destHost;

        pmDataTransferInfo() : memHandle(NULL), memLength(0), operatedMemLength(NULL), memType(MAX_MEM_TYPE), srcHost((uint)-1), destHost((uint)-1) {}
    } pmDataTransferInfo;

    typedef enum pmDeviceType
    {
        CPU = 0,
        GPU_CUDA,
        MAX_DEVICE_TYPES
    } pmDeviceType;

    typedef struct pmDeviceInfo
    {
        pmDeviceHandle deviceHandle;
        char name[MAX_NAME_STR_LEN];
        char description[MAX_DESC_STR_LEN];
        pmDeviceType deviceType;
        uint host;
        uint deviceIdOnHost;
        uint deviceIdInCluster;

        pmDeviceInfo() : deviceHandle(NULL), deviceType(MAX_DEVICE_TYPES), host((uint)-1), deviceIdOnHost((uint)-1), deviceIdInCluster((uint)-1)
        {
            name[0] = 0;
            description[0] = 0;
        }
    } pmDeviceInfo;

    typedef enum pmSchedulingPolicy
    {
        SLOW_START,
        RANDOM_STEAL,
        RANDOM_STEAL_WITH_AFFINITY,
        EQUAL_STATIC,
        PROPORTIONAL_STATIC,
        NODE_EQUAL_STATIC
    } pmSchedulingPolicy;

    typedef enum pmAffinityCriterion
    {
        MAXIMIZE_LOCAL_DATA,
        MINIMIZE_REMOTE_SOURCES,
        MINIMIZE_REMOTE_TRANSFER_EVENTS,
        MINIMIZE_REMOTE_TRANSFERS_ESTIMATED_TIME,
        DERIVED_AFFINITY,
        MAX_AFFINITY_CRITERION
    } pmAffinityCriterion;

    /* Lifetime of a per-subtask scratch buffer. */
    typedef enum pmScratchBufferType
    {
        PRE_SUBTASK_TO_SUBTASK,
        SUBTASK_TO_POST_SUBTASK,
        PRE_SUBTASK_TO_POST_SUBTASK,
        REDUCTION_TO_REDUCTION
    } pmScratchBufferType;

    typedef struct pmRedistributionMetadata
    {
        uint order;
        uint count;

        pmRedistributionMetadata() : order(0), count(0) {}
        pmRedistributionMetadata(uint pOrder, uint pCount) : order(pOrder), count(pCount) {}
    } pmRedistributionMetadata;

    /* User callbacks. */
    typedef pmStatus (*pmDataDistributionCallback)(pmTaskInfo pTaskInfo, pmDeviceInfo pDeviceInfo, pmSubtaskInfo pSubtaskInfo);
    typedef pmStatus (*pmSubtaskCallback_CPU)(pmTaskInfo pTaskInfo, pmDeviceInfo pDeviceInfo, pmSubtaskInfo pSubtaskInfo);
    typedef void (*pmSubtaskCallback_GPU_CUDA)(pmTaskInfo pTaskInfo, pmDeviceInfo* pDeviceInfo, pmSubtaskInfo pSubtaskInfo, pmStatus* pStatus);
    typedef pmStatus (*pmSubtaskCallback_GPU_Custom)(pmTaskInfo pTaskInfo, pmDeviceInfo pDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream);
    typedef pmStatus (*pmDataReductionCallback)(pmTaskInfo pTaskInfo, pmDeviceInfo pDevice1Info, pmSubtaskInfo pSubtask1Info, pmDeviceInfo pDevice2Info, pmSubtaskInfo pSubtask2Info);
    typedef pmStatus (*pmDataRedistributionCallback)(pmTaskInfo pTaskInfo, pmDeviceInfo pDeviceInfo, pmSubtaskInfo pSubtaskInfo);
    typedef bool (*pmDeviceSelectionCallback)(pmTaskInfo pTaskInfo, pmDeviceInfo pDeviceInfo);
    typedef pmStatus (*pmPreDataTransferCallback)(pmTaskInfo pTaskInfo, pmDataTransferInfo pDataTransferInfo);
    typedef pmStatus (*pmPostDataTransferCallback)(pmTaskInfo pTaskInfo, pmDataTransferInfo pDataTransferInfo);
    typedef pmStatus (*pmTaskCompletionCallback)(pmTaskInfo pTaskInfo);

    typedef struct pmCallbacks
    {
    public:
        pmDataDistributionCallback dataDistribution;
        pmSubtaskCallback_CPU subtask_cpu;
        pmSubtaskCallback_GPU_CUDA subtask_gpu_cuda;
        pmSubtaskCallback_GPU_Custom subtask_gpu_custom;    /* at most one of the two GPU callbacks may be set */
        pmDataReductionCallback dataReduction;
        pmDataRedistributionCallback dataRedistribution;
        pmDeviceSelectionCallback deviceSelection;
        pmPreDataTransferCallback preDataTransfer;
        pmPostDataTransferCallback postDataTransfer;
        pmTaskCompletionCallback taskCompletionCallback;
        const char* subtask_opencl;

        pmCallbacks() { Clear(); }
        pmCallbacks(pmDataDistributionCallback pDD, const char* pOpenCL) { Clear(); dataDistribution = pDD; subtask_opencl = pOpenCL; }
        pmCallbacks(pmDataDistributionCallback pDD, const char* pOpenCL, pmDataReductionCallback pRed) { Clear(); dataDistribution = pDD; subtask_opencl = pOpenCL; dataReduction = pRed; }
        pmCallbacks(pmDataDistributionCallback pDD, const char* pOpenCL, pmDataRedistributionCallback pRedist) { Clear(); dataDistribution = pDD; subtask_opencl = pOpenCL; dataRedistribution = pRedist; }
        pmCallbacks(pmDataDistributionCallback pDD, pmSubtaskCallback_CPU pCpu, pmSubtaskCallback_GPU_CUDA pCuda) { Clear(); dataDistribution = pDD; subtask_cpu = pCpu; subtask_gpu_cuda = pCuda; }
        pmCallbacks(pmDataDistributionCallback pDD, pmSubtaskCallback_CPU pCpu, pmSubtaskCallback_GPU_Custom pCustom) { Clear(); dataDistribution = pDD; subtask_cpu = pCpu; subtask_gpu_custom = pCustom; }
        pmCallbacks(pmDataDistributionCallback pDD, pmSubtaskCallback_CPU pCpu, pmSubtaskCallback_GPU_CUDA pCuda, pmDataReductionCallback pRed) { Clear(); dataDistribution = pDD; subtask_cpu = pCpu; subtask_gpu_cuda = pCuda; dataReduction = pRed; }
        pmCallbacks(pmDataDistributionCallback pDD, pmSubtaskCallback_CPU pCpu, pmSubtaskCallback_GPU_Custom pCustom, pmDataReductionCallback pRed) { Clear(); dataDistribution = pDD; subtask_cpu = pCpu; subtask_gpu_custom = pCustom; dataReduction = pRed; }
        pmCallbacks(pmDataDistributionCallback pDD, pmSubtaskCallback_CPU pCpu, pmSubtaskCallback_GPU_CUDA pCuda, pmDataRedistributionCallback pRedist) { Clear(); dataDistribution = pDD; subtask_cpu = pCpu; subtask_gpu_cuda = pCuda; dataRedistribution = pRedist; }
        pmCallbacks(pmDataDistributionCallback pDD, pmSubtaskCallback_CPU pCpu, pmSubtaskCallback_GPU_Custom pCustom, pmDataRedistributionCallback pRedist) { Clear(); dataDistribution = pDD; subtask_cpu = pCpu; subtask_gpu_custom = pCustom; dataRedistribution = pRedist; }

    private:
        void Clear()
        {
            dataDistribution = NULL; subtask_cpu = NULL; subtask_gpu_cuda = NULL; subtask_gpu_custom = NULL;
            dataReduction = NULL; dataRedistribution = NULL; deviceSelection = NULL; preDataTransfer = NULL;
            postDataTransfer = NULL; taskCompletionCallback = NULL; subtask_opencl = NULL;
        }
    } pmCallbacks;

    pmStatus pmRegisterCallbacks(const char* pKey, pmCallbacks pCallbacks, pmCallbackHandle* pCallbackHandle);
    pmStatus pmReleaseCallbacks(pmCallbackHandle pCallbackHandle);

    pmStatus pmCreateMemory(size_t pLength, pmMemHandle* pMemHandle);
    pmStatus pmCreateMemory2D(size_t pRows, size_t pCols, pmMemHandle* pMemHandle);
    pmStatus pmReleaseMemory(pmMemHandle pMemHandle);
    pmStatus pmFetchMemory(pmMemHandle pMemHandle);
    pmStatus pmFetchMemoryRange(pmMemHandle pMemHandle, size_t pOffset, size_t pLength);
    pmStatus pmGetRawMemPtr(pmMemHandle pMemHandle, pmRawMemPtr* pPtr);

    /* Callable only from a data-distribution callback. */
    pmStatus pmSubscribeToMemory(pmTaskHandle pTaskHandle, pmDeviceHandle pDeviceHandle, ulong pSubtaskId, pmSplitInfo& pSplitInfo, uint pMemIndex, pmSubscriptionType pSubscriptionType, const pmSubscriptionInfo& pSubscriptionInfo);
    pmStatus pmSubscribeToMemory(pmTaskHandle pTaskHandle, pmDeviceHandle pDeviceHandle, ulong pSubtaskId, pmSplitInfo& pSplitInfo, uint pMemIndex, pmSubscriptionType pSubscriptionType, const pmScatteredSubscriptionInfo& pScatteredSubscriptionInfo);

    /* Callable only from a data-redistribution callback. */
    pmStatus pmRedistributeData(pmTaskHandle pTaskHandle, pmDeviceHandle pDeviceHandle, ulong pSubtaskId, pmSplitInfo& pSplitInfo, uint pMemIndex, size_t pOffset, size_t pLength, uint pOrder);

    /* Kernel launch shape for a subtask_gpu_cuda subtask. */
    typedef struct pmCudaLaunchConf
    {
        int blocksX;
        int blocksY;
        int blocksZ;
        int threadsX;
        int threadsY;
        int threadsZ;
        int sharedMem;

        pmCudaLaunchConf() : blocksX(1), blocksY(1), blocksZ(1), threadsX(1), threadsY(1), threadsZ(1), sharedMem(0) {}
        pmCudaLaunchConf(int pBX, int pBY, int pBZ, int pTX, int pTY, int pTZ)
            : blocksX(pBX), blocksY(pBY), blocksZ(pBZ), threadsX(pTX), threadsY(pTY), threadsZ(pTZ), sharedMem(0) {}
        pmCudaLaunchConf(int pBX, int pBY, int pBZ, int pTX, int pTY, int pTZ, int pSharedMem)
            : blocksX(pBX), blocksY(pBY), blocksZ(pBZ), threadsX(pTX), threadsY(pTY), threadsZ(pTZ), sharedMem(pSharedMem) {}
    } pmCudaLaunchConf;

    /* Callable only from a data-distribution callback. */
    pmStatus pmSetCudaLaunchConf(pmTaskHandle pTaskHandle, pmDeviceHandle pDeviceHandle, ulong pSubtaskId, pmSplitInfo& pSplitInfo, pmCudaLaunchConf& pCudaLaunchConf);
    pmStatus pmReserveCudaGlobalMem(pmTaskHandle pTaskHandle, pmDeviceHandle pDeviceHandle, ulong pSubtaskId, pmSplitInfo& pSplitInfo, size_t pSize);

    typedef struct pmTaskMem
    {
        pmMemHandle memHandle;
        pmMemType memType;
        pmSubscriptionVisibilityType subscriptionVisibilityType;
        bool disjointReadWritesAcrossSubtasks;

        pmTaskMem() : memHandle(NULL), memType(MAX_MEM_TYPE), subscriptionVisibilityType(SUBSCRIPTION_NATURAL), disjointReadWritesAcrossSubtasks(false) {}
        pmTaskMem(pmMemHandle pHandle, pmMemType pType)
            : memHandle(pHandle), memType(pType), subscriptionVisibilityType(SUBSCRIPTION_NATURAL), disjointReadWritesAcrossSubtasks(false) {}
        pmTaskMem(pmMemHandle pHandle, pmMemType pType, pmSubscriptionVisibilityType pVis)
            : memHandle(pHandle), memType(pType), subscriptionVisibilityType(pVis), disjointReadWritesAcrossSubtasks(false) {}
        pmTaskMem(pmMemHandle pHandle, pmMemType pType, pmSubscriptionVisibilityType pVis, bool pDisjoint)
            : memHandle(pHandle), memType(pType), subscriptionVisibilityType(pVis), disjointReadWritesAcrossSubtasks(pDisjoint) {}
    } pmTaskMem;

    typedef struct pmTaskDetails
    {
        void* taskConf;
        uint taskConfLength;
        pmTaskMem* taskMem;
        uint taskMemCount;
        pmCallbackHandle callbackHandle;
        ulong subtaskCount;
        ulong taskId;
        ushort priority;
        pmSchedulingPolicy policy;
        int timeOutInSecs;                 /* negative: no timeout */
        bool multiAssignEnabled;
        bool overlapComputeCommunication;
        bool canSplitCpuSubtasks;
        bool canSplitGpuSubtasks;
        bool cudaCacheEnabled;
        bool suppressTaskLogs;
        pmAffinityCriterion affinityCriterion;
        pmClusterHandle cluster;

        pmTaskDetails()
            : taskConf(NULL), taskConfLength(0), taskMem(NULL), taskMemCount(0), callbackHandle(NULL), subtaskCount(0), taskId(0), priority(0),
              policy(RANDOM_STEAL), timeOutInSecs(INT_MAX), multiAssignEnabled(true), overlapComputeCommunication(true), canSplitCpuSubtasks(false),
              canSplitGpuSubtasks(false), cudaCacheEnabled(true), suppressTaskLogs(false), affinityCriterion(MAXIMIZE_LOCAL_DATA), cluster(NULL) {}
        pmTaskDetails(void* pTaskConf, uint pTaskConfLength, pmTaskMem* pTaskMem, uint pTaskMemCount, pmCallbackHandle pCallbackHandle, ulong pSubtaskCount)
            : taskConf(pTaskConf), taskConfLength(pTaskConfLength), taskMem(pTaskMem), taskMemCount(pTaskMemCount), callbackHandle(pCallbackHandle),
              subtaskCount(pSubtaskCount), taskId(0), priority(0), policy(RANDOM_STEAL), timeOutInSecs(INT_MAX), multiAssignEnabled(true),
              overlapComputeCommunication(true), canSplitCpuSubtasks(false), canSplitGpuSubtasks(false), cudaCacheEnabled(true), suppressTaskLogs(false),
              affinityCriterion(MAXIMIZE_LOCAL_DATA), cluster(NULL) {}
    } pmTaskDetails;

    pmStatus pmSubmitTask(pmTaskDetails pTaskDetails, pmTaskHandle* pTaskHandle);
    pmStatus pmReleaseTask(pmTaskHandle pTaskHandle);
    pmStatus pmWaitForTaskCompletion(pmTaskHandle pTaskHandle);
    pmStatus pmGetTaskExecutionTimeInSecs(pmTaskHandle pTaskHandle, double* pTime);
    pmStatus pmReleaseTaskAndResources(pmTaskDetails pTaskDetails, pmTaskHandle pTaskHandle);

    /* Scratch buffer shared by the callbacks of one subtask.  On the device it
     * is gpuContext->scratchBuffer; on the host the library allocates it on the
     * first request (later requests return the same buffer). */
#ifdef __CUDACC__
    __host__ __device__
#endif
    inline void* pmGetScratchBuffer(pmTaskHandle pTaskHandle, pmDeviceHandle pDeviceHandle, ulong pSubtaskId, pmSplitInfo& pSplitInfo, pmScratchBufferType pScratchBufferType, size_t pBufferSize, pmGpuContext* pGpuContext)
    {
#if defined(__CUDA_ARCH__)
        return (pGpuContext ? pGpuContext->scratchBuffer : NULL);
#else
        void* pmGetScratchBufferHostFunc(pmTaskHandle, pmDeviceHandle, ulong, pmSplitInfo&, pmScratchBufferType, size_t);
        return pmGetScratchBufferHostFunc(pTaskHandle, pDeviceHandle, pSubtaskId, pSplitInfo, pScratchBufferType, pBufferSize);
#endif
    }

    pmStatus pmReleaseScratchBuffer(pmTaskHandle pTaskHandle, pmDeviceHandle pDeviceHandle, ulong pSubtaskId, pmSplitInfo& pSplitInfo, pmScratchBufferType pScratchBufferType);
    void* pmGetLastReductionScratchBuffer(pmTaskHandle pTaskHandle);
    pmRedistributionMetadata* pmGetRedistributionMetadata(pmTaskHandle pTaskHandle, uint pMemIndex, ulong* pCount);

} // namespace pm

#endif
