/*
 * ref_lu_glue.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Drives the reference's own luDecomposition CPU code
 * (testSuite/luDecomposition/source/code/src/luDecomposition.cpp, compiled
 * unchanged by oracle/ref/Makefile against oracle/ref/cblas) on caller
 * buffers:
 *   - ref_lu_serial: serialLUDecomposition (:116-125), the unblocked,
 *     unpivoted column-major LU in Crout form (L keeps the diagonal, U is
 *     unit upper);
 *   - ref_lu_blocked: the app's task sequence of DoParallelProcess
 *     (:440-463) -- per block step, LU_DECOMPOSE (1 subtask), HORZ_VERT_COMP
 *     (2 (nb - k - 1) subtasks), DIAGONAL_COMP ((nb - k - 1)^2 subtasks), and a
 *     last LU_DECOMPOSE -- each subtask through its data distribution
 *     callback (subscriptions recorded) and its CPU callback on NATURAL views,
 *     with pTaskInfo.taskId = k as StageParallelTask sets it (:413-425).
 * Subtasks run one after another; the BLAS threads each call.
 */
#include <cstdint>

#include "commonAPI.h"
#include "luDecomposition.h"
#include "ref_blas_stubs.h"

namespace luDecomposition {
void serialLUDecomposition(MATRIX_DATA_TYPE*, size_t, size_t);
pmStatus luDecompositionDataDistribution(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
pmStatus luDecomposition_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
pmStatus horizVertCompDataDistribution(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
pmStatus horizVertComp_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
pmStatus diagCompDataDistribution(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
pmStatus diagComp_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
}  // namespace luDecomposition

using namespace luDecomposition;

namespace {
typedef pmStatus (*Cb)(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);

int run_stage(Cb dd, Cb cpu, float* A, size_t n, size_t task, unsigned long subtasks) {
    luTaskConf conf;
    conf.matrixDim = n;
    pmTaskInfo ti;
    ti.taskConf = &conf;
    ti.taskConfLength = sizeof(conf);
    ti.taskId = task;
    ti.subtaskCount = subtasks;
    pmDeviceInfo di;
    di.deviceType = pm::CPU;
    for (unsigned long id = 0; id < subtasks; ++id) {
        pmSubtaskInfo si;
        si.subtaskId = id;
        refglue::t_subs.clear();
        if (dd(ti, di, si) != pmSuccess) return 1;
        const size_t lo = refglue::lowest(OUTPUT_MEM_INDEX);
        if (lo == (size_t)-1) return 2;
        void* p = (char*)A + lo;
        si.memCount = MAX_MEM_INDICES;
        si.memInfo[OUTPUT_MEM_INDEX] = pmMemInfo(p, p, p, 0, SUBSCRIPTION_NATURAL);
        if (cpu(ti, di, si) != pmSuccess) return 3;
    }
    return 0;
}
}  // namespace

extern "C" {

/* BLOCK_DIM of luDecomposition.h this library was compiled with. */
unsigned long ref_lu_block_dim(void) { return BLOCK_DIM; }

/* In-place serialLUDecomposition of the leading n x n block of a
 * column-major matrix with column stride ld (elements). */
int ref_lu_serial(float* A, unsigned long n, unsigned long ld) {
    if (n < 1 || ld < n) return 1;
    serialLUDecomposition(A, n, ld);
    return 0;
}

/* In-place blocked LU of a column-major n x n matrix (ld = n), n a multiple of
 * BLOCK_DIM, by the reference app's three stages.  Returns 0 on success. */
int ref_lu_blocked(float* A, unsigned long n) {
    if (n < BLOCK_DIM || n % BLOCK_DIM) return 4;
    const size_t nb = n / BLOCK_DIM;
    for (size_t k = 0; k + 1 < nb; ++k) {
        int st = run_stage(luDecompositionDataDistribution, luDecomposition_cpu, A, n, k, 1);
        if (!st) st = run_stage(horizVertCompDataDistribution, horizVertComp_cpu, A, n, k, 2 * (nb - k - 1));
        if (!st) st = run_stage(diagCompDataDistribution, diagComp_cpu, A, n, k, (nb - k - 1) * (nb - k - 1));
        if (st) return st;
    }
    return run_stage(luDecompositionDataDistribution, luDecomposition_cpu, A, n, nb - 1, 1);
}
}
