// B200 GPU callbacks of the matrixMultiplyBlas app: a drop-in replacement for
// testSuite/matrixMultiplyBlas/source/code/src/matrixMultiplyBlasCUDA.cu.
//
// matrixMultiply_cudaLaunchFunc keeps the reference callback's contract
// (:54-77): C block = A row block x B column block, row-major fp32, with the
// B/C leading dimensions n (NATURAL view) or blockDim (COMPACT view); the
// product runs on the tcgen05 BF16x3 kernel instead of cublasSgemm.  The split
// buffers the kernel needs are cached per stream, so a callback allocates
// only when a stream first sees a larger problem.
//
// A batch hook lets the runtime run the subtasks of a task (NATURAL views) in
// groups: the C blocks of a group are one grouped product launch
// (pmb_sgemm_bf16x3_grouped) instead of one split + product launch pair per
// subtask.  Two groups per task, so the second group's staging overlaps the
// first group's products.
#include "matrixMultiplyBlas_b200.h"

#include <map>
#include <mutex>
#include <vector>

#include "pmb_capi.h"

extern "C" int pmb_runtime_register_batch_groups(void* subtask_gpu_custom, void* batch_fn, int groups);

namespace matrixMultiplyBlas {

using namespace pm;

namespace {

struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
};

std::mutex g_mu;
std::map<void*, Workspace> g_ws;  // per stream

int workspace_for(void* stream, size_t need, void** out) {
    std::lock_guard<std::mutex> g(g_mu);
    Workspace& w = g_ws[stream];
    if (w.bytes < need) {
        if (w.ptr) {
            const int st = pmb_stream_synchronize(stream);  // the old buffer may still be in use
            if (st != PMB_SUCCESS) return st;
            pmb_free(w.ptr);
        }
        w.ptr = nullptr;
        w.bytes = 0;
        const int st = pmb_malloc(&w.ptr, need);
        if (st != PMB_SUCCESS) return st;
        w.bytes = need;
    }
    *out = w.ptr;
    return PMB_SUCCESS;
}

// The C block of one subtask as a product (false: the subtask has no block).
bool problem_for(const matrixMultiplyTaskConf* conf, const pmSubtaskInfo& si, pmb_gemm_problem& q) {
    size_t offset = 0, height = 0;
    pmSplitInfo split = si.splitInfo;
    if (!GetSplitData(&offset, &height, const_cast<matrixMultiplyTaskConf*>(conf), split)) return false;
    const int n = static_cast<int>(conf->matrixDim), bd = static_cast<int>(conf->blockDim);
    const pmMemInfo& a = si.memInfo[kMatrixA];
    const pmMemInfo& b = si.memInfo[kMatrixB];
    const pmMemInfo& c = si.memInfo[kMatrixC];
    q.M = static_cast<int>(height);
    q.N = bd;
    q.K = n;
    q.alpha = 1.0f;
    q.A = static_cast<const float*>(a.ptr);
    q.lda = n;
    q.B = static_cast<const float*>(b.ptr);
    q.ldb = b.visibilityType == SUBSCRIPTION_NATURAL ? n : bd;
    q.beta = 0.0f;
    q.C = static_cast<float*>(c.ptr);
    q.ldc = c.visibilityType == SUBSCRIPTION_NATURAL ? n : bd;
    return true;
}

pmStatus matrixMultiply_batch(const pmTaskInfo* task, const pmDeviceInfo*, const pmSubtaskInfo* subtasks,
                              unsigned long count, void* stream) {
    const matrixMultiplyTaskConf* conf = static_cast<const matrixMultiplyTaskConf*>(task->taskConf);
    std::vector<pmb_gemm_problem> probs;
    probs.reserve(count);
    for (unsigned long i = 0; i < count; ++i) {
        pmb_gemm_problem q;
        if (problem_for(conf, subtasks[i], q)) probs.push_back(q);
    }
    if (probs.empty()) return pmSuccess;
    const size_t need = pmb_gemm_grouped_workspace_bytes(probs.data(), static_cast<int>(probs.size()));
    void* ws = nullptr;
    int st = workspace_for(stream, need, &ws);
    if (st == PMB_SUCCESS)
        st = pmb_sgemm_bf16x3_grouped(probs.data(), static_cast<int>(probs.size()), ws, need, stream);
    return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st);
}

struct Registrar {
    Registrar() {
        pmb_runtime_register_batch_groups(reinterpret_cast<void*>(&matrixMultiply_cudaLaunchFunc),
                                          reinterpret_cast<void*>(&matrixMultiply_batch), 2);
    }
} g_registrar;

}  // namespace

pmStatus matrixMultiply_cudaLaunchFunc(pmTaskInfo pTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream) {
    matrixMultiplyTaskConf* conf = static_cast<matrixMultiplyTaskConf*>(pTaskInfo.taskConf);
    size_t offset = 0, height = 0;
    if (!GetSplitData(&offset, &height, conf, pSubtaskInfo.splitInfo)) return pmSuccess;
    const int n = static_cast<int>(conf->matrixDim), bd = static_cast<int>(conf->blockDim);
    const pmMemInfo& a = pSubtaskInfo.memInfo[kMatrixA];
    const pmMemInfo& b = pSubtaskInfo.memInfo[kMatrixB];
    const pmMemInfo& c = pSubtaskInfo.memInfo[kMatrixC];
    const int64_t ldb = b.visibilityType == SUBSCRIPTION_NATURAL ? n : bd;
    const int64_t ldc = c.visibilityType == SUBSCRIPTION_NATURAL ? n : bd;
    const size_t need = pmb_gemm_workspace_bytes(static_cast<int>(height), bd, n);
    void* ws = nullptr;
    int st = workspace_for(pCudaStream, need, &ws);
    if (st == PMB_SUCCESS)
        st = pmb_sgemm_bf16x3(static_cast<int>(height), bd, n, 1.0f, static_cast<const float*>(a.ptr), n,
                              static_cast<const float*>(b.ptr), ldb, 0.0f, static_cast<float*>(c.ptr), ldc, ws, need,
                              pCudaStream);
    return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st);
}

int singleGpuMatrixMultiply(float* pInputMatrices, float* pOutputMatrix, int pDim) {
    const size_t elems = static_cast<size_t>(pDim) * pDim;
    void *d_in = nullptr, *d_out = nullptr, *ws = nullptr, *s = nullptr;
    const size_t wsb = pmb_gemm_workspace_bytes(pDim, pDim, pDim);
    int st = pmb_malloc(&d_in, 8 * elems);
    if (st == PMB_SUCCESS) st = pmb_malloc(&d_out, 4 * elems);
    if (st == PMB_SUCCESS) st = pmb_malloc(&ws, wsb);
    if (st == PMB_SUCCESS) st = pmb_stream_create(&s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(d_in, pInputMatrices, 8 * elems, PMB_H2D, s);
    const float* A = static_cast<const float*>(d_in);
    if (st == PMB_SUCCESS)
        st = pmb_sgemm_bf16x3(pDim, pDim, pDim, 1.0f, A, pDim, A + elems, pDim, 0.0f, static_cast<float*>(d_out), pDim,
                              ws, wsb, s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(pOutputMatrix, d_out, 4 * elems, PMB_D2H, s);
    if (st == PMB_SUCCESS) st = pmb_stream_synchronize(s);
    pmb_stream_destroy(s);
    pmb_free(ws);
    pmb_free(d_out);
    pmb_free(d_in);
    return st == PMB_SUCCESS ? 0 : 1;
}

}  // namespace matrixMultiplyBlas

// The reference harness frees its cuBLAS handles at exit (commonAPI.cpp:291-296);
// the B200 callbacks hold none.
void FreeCublasHandles() {}
