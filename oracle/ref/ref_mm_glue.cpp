/*
 * ref_mm_glue.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Drives the reference's own matrixMultiplyBlas CPU callbacks
 * (testSuite/matrixMultiplyBlas/source/code/src/matrixMultiplyBlas.cpp,
 * compiled unchanged by oracle/ref/Makefile against oracle/ref/cblas) on
 * caller buffers: for each subtask, matrixMultiplyDataDistribution (:90-113)
 * records its three scattered subscriptions, and matrixMultiply_cpu
 * (:115-133) runs on NATURAL views of them, as the reference runtime's CPU
 * stub would.  Subtasks run one after another; the BLAS threads each GEMM.
 */
#include <cstdint>

#include "commonAPI.h"
#include "matrixMultiplyBlas.h"
#include "ref_blas_stubs.h"

namespace matrixMultiplyBlas {
pmStatus matrixMultiplyDataDistribution(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
pmStatus matrixMultiply_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
size_t getBlockSize(size_t);
}  // namespace matrixMultiplyBlas

using namespace matrixMultiplyBlas;

extern "C" {

/* BLOCK_DIM of matrixMultiplyBlas.h this library was compiled with. */
int ref_mm_block_dim(void) { return BLOCK_DIM; }

/* The reference app's block size for an n x n product (getBlockSize, :52-55). */
unsigned long ref_mm_block_size(unsigned long n) { return getBlockSize(n); }

/* Subscriptions of subtask `id` of an n x n product in blocks of `block`:
 * out[mem * 5 + {0..4}] = {type, offset, size, step, count} for the three
 * memory indices (A, B, C).  Returns 0, or 1 if a memory index has no
 * subscription or more than one. */
int ref_mm_subscriptions(unsigned long n, unsigned long block, unsigned long id, unsigned long long* out) {
    matrixMultiplyTaskConf conf;
    conf.matrixDim = n;
    conf.blockDim = block;
    pmTaskInfo ti;
    ti.taskConf = &conf;
    ti.taskConfLength = sizeof(conf);
    ti.subtaskCount = (n / block) * (n / block);
    pmDeviceInfo di;
    di.deviceType = pm::CPU;
    pmSubtaskInfo si;
    si.subtaskId = id;
    refglue::t_subs.clear();
    if (matrixMultiplyDataDistribution(ti, di, si) != pmSuccess) return 2;
    for (unsigned m = 0; m < MAX_MEM_INDICES; ++m) {
        int found = 0;
        for (const refglue::Sub& s : refglue::t_subs)
            if (s.mem == m) {
                ++found;
                out[m * 5 + 0] = (unsigned long long)s.type;
                out[m * 5 + 1] = s.info.offset;
                out[m * 5 + 2] = s.info.size;
                out[m * 5 + 3] = s.info.step;
                out[m * 5 + 4] = s.info.count;
            }
        if (found != 1) return 1;
    }
    return 0;
}

/* C = A * B (row-major n x n fp32) as the reference's task of (n/block)^2
 * subtasks computes it.  Returns 0 on success. */
int ref_mm_task(const float* A, const float* B, float* C, unsigned long n, unsigned long block) {
    if (!block || n % block) return 4;
    matrixMultiplyTaskConf conf;
    conf.matrixDim = n;
    conf.blockDim = block;
    pmTaskInfo ti;
    ti.taskConf = &conf;
    ti.taskConfLength = sizeof(conf);
    ti.subtaskCount = (n / block) * (n / block);
    pmDeviceInfo di;
    di.deviceType = pm::CPU;
    char* base[MAX_MEM_INDICES] = {(char*)A, (char*)B, (char*)C};
    for (unsigned long id = 0; id < ti.subtaskCount; ++id) {
        pmSubtaskInfo si;
        si.subtaskId = id;
        refglue::t_subs.clear();
        if (matrixMultiplyDataDistribution(ti, di, si) != pmSuccess) return 1;
        si.memCount = MAX_MEM_INDICES;
        for (unsigned m = 0; m < MAX_MEM_INDICES; ++m) {
            const size_t lo = refglue::lowest(m);
            if (lo == (size_t)-1) return 2;
            void* p = base[m] + lo;
            si.memInfo[m] = m == OUTPUT_MATRIX_MEM_INDEX ? pmMemInfo(p, NULL, p, 0, SUBSCRIPTION_NATURAL)
                                                         : pmMemInfo(p, p, NULL, 0, SUBSCRIPTION_NATURAL);
        }
        if (matrixMultiply_cpu(ti, di, si) != pmSuccess) return 3;
    }
    return 0;
}
}
