/*
 * ref_lu_gpu_glue.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference luDecomposition app's own parallel driver,
 * DoParallelProcess (testSuite/luDecomposition/source/code/src/
 * luDecomposition.cpp:425-470; compiled unchanged with BUILD_CUDA by
 * oracle/ref/Makefile), on a caller matrix: per block step its three stage
 * tasks (LU_DECOMPOSE, HORZ_VERT_COMP, DIAGONAL_COMP) are submitted through
 * the B200 pm:: runtime (libpmlib.so) with the app's own callback sets
 * (DoSetDefaultCallbacks1-3: its data distributions and the GPU callbacks
 * of libpmb_app_luDecomposition.so), then the address space is fetched back.
 * The commonAPI helpers the app's task code calls are given their default
 * values here (the app's harness, commonAPI.cpp, owns main and the argument
 * parsing, which this glue replaces).
 */
#include <chrono>
#include <cstdio>

#include "commonAPI.h"
#include "luDecomposition.h"

namespace luDecomposition {
extern MATRIX_DATA_TYPE* gParallelOutput;
double DoParallelProcess(int argc, char** argv, int pCommonArgs, pmCallbackHandle* pCallbackHandle,
                         pmSchedulingPolicy pSchedulingPolicy, bool pFetchBack);
pmCallbacks DoSetDefaultCallbacks1();
pmCallbacks DoSetDefaultCallbacks2();
pmCallbacks DoSetDefaultCallbacks3();
}  // namespace luDecomposition

bool isMultiAssignEnabled() { return false; }
uint getAffinityCriterion() { return 0; }
bool isComputeCommunicationOverlapEnabled() { return true; }
bool isLazyMemEnabled() { return false; }
bool isCudaCacheEnabled() { return true; }
double getCurrentTimeInSecs() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
void DistributeMemory(pmMemHandle, memDistributionType, unsigned int, unsigned int, unsigned int, unsigned int, bool) {}
void commonStart(int, char**, initFunc, serialProcessFunc, singleGpuProcessFunc, parallelProcessFunc, compareFunc,
                 destroyFunc, callbackStruct*, size_t) {}
void commonFinish() {}

extern "C" {

/* In-place LU of the column-major n x n matrix A (n a multiple of BLOCK_DIM)
 * by the app's DoParallelProcess on the B200 runtime.  Returns 0 on success. */
int ref_lu_app_gpu(float* A, unsigned long n) {
    using namespace luDecomposition;
    if (n < BLOCK_DIM || n % BLOCK_DIM) return 4;
    if (pmInitialize() != pmSuccess) return 1;
    static pmCallbackHandle handles[3] = {nullptr, nullptr, nullptr};
    if (!handles[0]) {
        if (pmRegisterCallbacks("LU_S1", DoSetDefaultCallbacks1(), &handles[0]) != pmSuccess ||
            pmRegisterCallbacks("LU_S2", DoSetDefaultCallbacks2(), &handles[1]) != pmSuccess ||
            pmRegisterCallbacks("LU_S3", DoSetDefaultCallbacks3(), &handles[2]) != pmSuccess)
            return 2;
    }
    gParallelOutput = A;
    char a0[] = "luDecomposition";
    char a1[32];
    std::snprintf(a1, sizeof(a1), "%lu", n);
    char* argv[] = {a0, a1};
    const double t = DoParallelProcess(2, argv, 0, handles, SLOW_START, true);
    return t > 0.0 ? 0 : 3;
}
}
