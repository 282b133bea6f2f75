// B200 GPU callbacks of the luDecomposition app: a drop-in replacement for
// testSuite/luDecomposition/source/code/src/luDecompositionCUDA.cu.
//
// Each callback keeps the reference callback's contract -- the same blocks,
// found at the same offsets from the subscription view (NATURAL: column stride
// matrixDim; COMPACT: the packed blocks), the same arithmetic result -- and
// enqueues its work on the subtask's stream only:
//   luDecomposition_cudaLaunchFunc (:66-97)  Crout LU of the diagonal block
//       (L keeps the pivots, U unit upper) by pmb_lu_decompose: FP64 64 x 64
//       diagonal factors and panel solves, BF16x3 tensor-core updates -- in
//       place of 2047 x {1-thread reciprocal kernel, cublasSscal, cublasSger};
//   horizVertComp_cudaLaunchFunc (:99-151)   U01 = L00^-1 A01 (left, lower,
//       non-unit) or L10 = A10 U00^-1 (right, upper, unit) by pmb_trsm_f32;
//   diagComp_cudaLaunchFunc (:153-193)       A11 -= L10 U01 by the BF16x3
//       tensor-core GEMM in place of cublasSgemm.
// The device workspaces are cached per stream, so a callback allocates only
// when its stream first needs a larger buffer.
#include "luDecomposition_b200.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

#include "pmb_capi.h"

namespace luDecomposition {

using namespace pm;

namespace {

constexpr int kNb = 64;

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

pmStatus to_pm(int st) { return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st); }

}  // namespace

pmStatus luDecomposition_cudaLaunchFunc(pmTaskInfo pTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo,
                                        void* pCudaStream) {
    const luTaskConf* conf = static_cast<const luTaskConf*>(pTaskInfo.taskConf);
    const pmMemInfo& mi = pSubtaskInfo.memInfo[kOutputMemIndex];
    float* block = static_cast<float*>(mi.ptr);
    const int64_t ld = mi.visibilityType == SUBSCRIPTION_NATURAL ? static_cast<int64_t>(conf->matrixDim)
                                                                 : static_cast<int64_t>(kBlockDim);
    const int n = static_cast<int>(kBlockDim);
    const size_t need = pmb_lu_workspace_bytes(n, kNb);
    void* ws = nullptr;
    int st = workspace_for(pCudaStream, need, &ws);
    if (st == PMB_SUCCESS) st = pmb_lu_decompose(block, n, ld, kNb, ws, need, pCudaStream);
    return to_pm(st);
}

pmStatus horizVertComp_cudaLaunchFunc(pmTaskInfo pTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo,
                                      void* pCudaStream) {
    const luTaskConf* conf = static_cast<const luTaskConf*>(pTaskInfo.taskConf);
    const pmMemInfo& mi = pSubtaskInfo.memInfo[kOutputMemIndex];
    const bool natural = mi.visibilityType == SUBSCRIPTION_NATURAL;
    const size_t n = conf->matrixDim, k = pTaskInfo.taskId;
    float* diag = static_cast<float*>(mi.ptr);  // block (k, k): the view's first subscribed element
    const int bd = static_cast<int>(kBlockDim);
    const bool upper = pSubtaskInfo.subtaskId < pTaskInfo.subtaskCount / 2;
    size_t offset;
    int64_t span;
    int side, uplo, unit;
    if (upper) {  // U01 = L00^-1 A01, A01 = block (k, k + 1 + id)
        offset = natural ? block_offset(k, k + 1 + pSubtaskInfo.subtaskId, n) - block_offset(k, k, n)
                         : kBlockDim * kBlockDim;
        span = natural ? static_cast<int64_t>(n) : bd;
        side = PMB_SIDE_LEFT;
        uplo = PMB_FILL_LOWER;
        unit = PMB_DIAG_NON_UNIT;
    } else {  // L10 = A10 U00^-1, A10 = block (k + 1 + id - half, k)
        const size_t first = pTaskInfo.subtaskCount / 2;
        offset = natural ? block_offset(k + 1 + pSubtaskInfo.subtaskId - first, k, n) - block_offset(k, k, n)
                         : kBlockDim;
        span = natural ? static_cast<int64_t>(n) : 2 * static_cast<int64_t>(bd);
        side = PMB_SIDE_RIGHT;
        uplo = PMB_FILL_UPPER;
        unit = PMB_DIAG_UNIT;
    }
    const size_t need = pmb_trsm_workspace_bytes(side, bd, bd);
    void* ws = nullptr;
    int st = workspace_for(pCudaStream, need, &ws);
    if (st == PMB_SUCCESS)
        st = pmb_trsm_f32(side, uplo, unit, bd, bd, diag, span, diag + offset, span, ws, need, pCudaStream);
    return to_pm(st);
}

pmStatus diagComp_cudaLaunchFunc(pmTaskInfo pTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream) {
    const luTaskConf* conf = static_cast<const luTaskConf*>(pTaskInfo.taskConf);
    const pmMemInfo& mi = pSubtaskInfo.memInfo[kOutputMemIndex];
    const bool natural = mi.visibilityType == SUBSCRIPTION_NATURAL;
    const size_t n = conf->matrixDim, k = pTaskInfo.taskId;
    const size_t dim = static_cast<size_t>(std::llround(std::sqrt(static_cast<double>(pTaskInfo.subtaskCount))));
    const size_t row = pSubtaskInfo.subtaskId / dim, col = pSubtaskInfo.subtaskId % dim;
    const int bd = static_cast<int>(kBlockDim);
    size_t off1, off2;
    int64_t span1, span2, span3;
    if (natural) {
        off1 = block_offset(k, k + 1 + col, n) - block_offset(k + 1 + row, k, n);
        off2 = block_offset(k + 1 + row, k + 1 + col, n) - block_offset(k + 1 + row, k, n);
        span1 = span2 = span3 = static_cast<int64_t>(n);
    } else {
        off1 = kBlockDim * kBlockDim;
        off2 = kBlockDim * kBlockDim + kBlockDim;
        span1 = bd;
        span2 = span3 = 2 * static_cast<int64_t>(bd);
    }
    float* L10 = static_cast<float*>(mi.ptr);  // block (k + 1 + row, k): the view's first subscribed element
    const float* U01 = L10 + off1;
    float* A11 = L10 + off2;
    const size_t need = pmb_gemm_workspace_bytes(bd, bd, bd);
    void* ws = nullptr;
    int st = workspace_for(pCudaStream, need, &ws);
    // A11 -= L10 U01 (column-major) == row-major A11^T -= U01^T L10^T.
    if (st == PMB_SUCCESS)
        st = pmb_sgemm_bf16x3(bd, bd, bd, -1.0f, U01, span2, L10, span1, 1.0f, A11, span3, ws, need, pCudaStream);
    return to_pm(st);
}

int singleGpuLUDecomposition(float* pMatrix, size_t pDim) {
    const int n = static_cast<int>(pDim);
    const size_t bytes = pDim * pDim * sizeof(float);
    const size_t wsb = pmb_lu_workspace_bytes(n, kNb);
    void *d = nullptr, *ws = nullptr, *s = nullptr;
    int st = pmb_malloc(&d, bytes);
    if (st == PMB_SUCCESS) st = pmb_malloc(&ws, wsb);
    if (st == PMB_SUCCESS) st = pmb_stream_create(&s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(d, pMatrix, bytes, PMB_H2D, s);
    if (st == PMB_SUCCESS) st = pmb_lu_decompose(static_cast<float*>(d), n, n, kNb, ws, wsb, s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(pMatrix, d, bytes, PMB_D2H, s);
    if (st == PMB_SUCCESS) st = pmb_stream_synchronize(s);
    pmb_stream_destroy(s);
    pmb_free(ws);
    pmb_free(d);
    return st == PMB_SUCCESS ? 0 : 1;
}

}  // namespace luDecomposition

// The reference harness frees its cuBLAS handles at exit (commonAPI.cpp:291-296);
// the B200 callbacks hold none.
void FreeCublasHandles() {}
