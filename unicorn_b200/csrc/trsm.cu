// Triangular solves of the luDecomposition app's HORZ_VERT_COMP stage, fp32
// column-major in place, alpha = 1 (the reference calls cublasStrsm,
// testSuite/luDecomposition/source/code/src/luDecompositionCUDA.cu:99-151, and
// cblas_strsm on the CPU, luDecomposition.cpp:216-275):
//   left  / lower / no transpose: B <- L^-1 B   (L m x m, B m x n): U01 = L00^-1 A01
//   right / upper / no transpose: B <- B U^-1   (U n x n, B m x n): L10 = A10 U00^-1
// each with a unit or a non-unit diagonal.
//
// Blocked right-looking solve over 64-wide diagonal blocks: the block's
// triangle is staged in shared memory in FP64 and every column (left) or row
// (right) of the panel is solved by one warp with FP64 substitution (lane l
// holds unknowns l and l + 32; each finished unknown is broadcast by a
// shuffle); the rest of B is then updated with the solved panel on the tensor
// cores (BF16x3 GEMM, K = 64): for the left solve B[k1:, :] -= L[k1:, k] X_k,
// for the right solve B[:, k1:] -= X_k U[k, k1:].
#include <algorithm>

#include "pmb_common.cuh"

extern "C" size_t pmb_gemm_workspace_bytes(int M, int N, int K);
namespace pmb {
int sgemm_bf16x3_launch(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                        float beta, float* C, int64_t ldc, void* workspace, size_t ws_bytes, cudaStream_t s,
                        bool clear_error);
}

namespace {

constexpr int kNb = 64;

// X_k = L_kk^-1 B_k for the kb rows k0.. of B (each of the `ncols` columns by
// one warp).  L_kk: rows/columns k0..k0+kb of A, lower, diagonal unit or not.
template <bool UNIT>
__global__ void __launch_bounds__(256)
trsm_left_lower_block(const float* __restrict__ A, int64_t lda, float* __restrict__ B, int64_t ldb, int k0, int kb,
                      int ncols) {
    __shared__ double sL[kNb * kNb];  // sL[c * 64 + r] = L(r, c), r > c; 0 elsewhere
    __shared__ double sInv[kNb];
    for (int e = threadIdx.x; e < kNb * kNb; e += 256) {
        const int c = e / kNb, r = e - c * kNb;
        const bool in = r < kb && c < kb;
        const double v = in ? static_cast<double>(A[static_cast<int64_t>(k0 + c) * lda + k0 + r]) : 0.0;
        sL[e] = r > c ? v : 0.0;
        if (r == c) sInv[r] = UNIT || !in ? 1.0 : 1.0 / v;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = 256 / 32;
    for (int col = blockIdx.x * wpb + (threadIdx.x >> 5); col < ncols; col += gridDim.x * wpb) {
        float* x = B + static_cast<int64_t>(col) * ldb + k0;
        double x0 = lane < kb ? static_cast<double>(x[lane]) : 0.0;
        double x1 = lane + 32 < kb ? static_cast<double>(x[lane + 32]) : 0.0;
#pragma unroll 8
        for (int i = 0; i < kNb; ++i) {
            const double xi = __shfl_sync(0xffffffffu, i < 32 ? x0 : x1, i & 31) * sInv[i];
            if (lane == (i & 31)) {
                if (i < 32) x0 = xi; else x1 = xi;
            }
            if (lane > i) x0 -= sL[i * kNb + lane] * xi;
            if (lane + 32 > i) x1 -= sL[i * kNb + lane + 32] * xi;
        }
        if (lane < kb) x[lane] = static_cast<float>(x0);
        if (lane + 32 < kb) x[lane + 32] = static_cast<float>(x1);
    }
}

// X_k = B_k U_kk^-1 for the kb columns k0.. of B (each of the `nrows` rows by
// one warp).  U_kk: rows/columns k0..k0+kb of A, upper, diagonal unit or not.
template <bool UNIT>
__global__ void __launch_bounds__(256)
trsm_right_upper_block(const float* __restrict__ A, int64_t lda, float* __restrict__ B, int64_t ldb, int k0, int kb,
                       int nrows) {
    __shared__ double sU[kNb * kNb];  // sU[r * 64 + c] = U(r, c), r < c; 0 elsewhere
    __shared__ double sInv[kNb];
    for (int e = threadIdx.x; e < kNb * kNb; e += 256) {
        const int c = e / kNb, r = e - c * kNb;  // consecutive threads read consecutive rows of a column
        const bool in = r < kb && c < kb;
        const double v = in ? static_cast<double>(A[static_cast<int64_t>(k0 + c) * lda + k0 + r]) : 0.0;
        sU[r * kNb + c] = r < c ? v : 0.0;
        if (r == c) sInv[r] = UNIT || !in ? 1.0 : 1.0 / v;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = 256 / 32;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < nrows; row += gridDim.x * wpb) {
        float* x = B + static_cast<int64_t>(k0) * ldb + row;  // element c of the panel row at x[c * ldb]
        double x0 = lane < kb ? static_cast<double>(x[static_cast<int64_t>(lane) * ldb]) : 0.0;
        double x1 = lane + 32 < kb ? static_cast<double>(x[static_cast<int64_t>(lane + 32) * ldb]) : 0.0;
#pragma unroll 8
        for (int c = 0; c < kNb; ++c) {
            const double xc = __shfl_sync(0xffffffffu, c < 32 ? x0 : x1, c & 31) * sInv[c];
            if (lane == (c & 31)) {
                if (c < 32) x0 = xc; else x1 = xc;
            }
            if (lane > c) x0 -= xc * sU[c * kNb + lane];
            if (lane + 32 > c) x1 -= xc * sU[c * kNb + lane + 32];
        }
        if (lane < kb) x[static_cast<int64_t>(lane) * ldb] = static_cast<float>(x0);
        if (lane + 32 < kb) x[static_cast<int64_t>(lane + 32) * ldb] = static_cast<float>(x1);
    }
}

int solve_grid(int items) { return std::max(1, std::min((items + 7) / 8, 4 * 148)); }

}  // namespace

extern "C" size_t pmb_trsm_workspace_bytes(int side, int m, int n) {
    if (m <= 0 || n <= 0) return 256;
    // The largest trailing update: the first step's.
    return side == PMB_SIDE_LEFT ? pmb_gemm_workspace_bytes(n, std::max(m - kNb, 1), kNb)
                                 : pmb_gemm_workspace_bytes(std::max(n - kNb, 1), m, kNb);
}

extern "C" int pmb_trsm_f32(int side, int uplo, int diag, int m, int n, const float* d_A, int64_t lda, float* d_B,
                            int64_t ldb, void* d_workspace, size_t ws_bytes, void* stream) {
    PMB_CHECK_ARG(side == PMB_SIDE_LEFT || side == PMB_SIDE_RIGHT, "bad side %d", side);
    PMB_CHECK_ARG((side == PMB_SIDE_LEFT && uplo == PMB_FILL_LOWER) || (side == PMB_SIDE_RIGHT && uplo == PMB_FILL_UPPER),
                  "only left/lower and right/upper solves are provided");
    PMB_CHECK_ARG(diag == PMB_DIAG_UNIT || diag == PMB_DIAG_NON_UNIT, "bad diagonal kind %d", diag);
    PMB_CHECK_ARG(m >= 0 && n >= 0, "negative size");
    if (m == 0 || n == 0) return PMB_SUCCESS;
    const int order = side == PMB_SIDE_LEFT ? m : n;
    PMB_CHECK_ARG(d_A && d_B && d_workspace, "null pointer");
    PMB_CHECK_ARG(lda >= order && ldb >= m, "leading dimensions too small");
    PMB_CHECK_ARG((reinterpret_cast<uintptr_t>(d_workspace) & 255) == 0, "workspace must be 256-byte aligned");
    PMB_CHECK_ARG(ws_bytes >= pmb_trsm_workspace_bytes(side, m, n), "TRSM workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool unit = diag == PMB_DIAG_UNIT;
    bool first = true;
    for (int k0 = 0; k0 < order; k0 += kNb) {
        const int kb = std::min(kNb, order - k0);
        const int rest = order - k0 - kb;
        int st;
        if (side == PMB_SIDE_LEFT) {
            if (unit) trsm_left_lower_block<true><<<solve_grid(n), 256, 0, s>>>(d_A, lda, d_B, ldb, k0, kb, n);
            else trsm_left_lower_block<false><<<solve_grid(n), 256, 0, s>>>(d_A, lda, d_B, ldb, k0, kb, n);
            PMB_CUDA_TRY(cudaGetLastError());
            if (rest == 0) break;
            // B[k1:, :] -= L[k1:, k] X_k (column-major) == row-major C^T -= X_k^T L^T: M = n, N = rest, K = kb
            st = pmb::sgemm_bf16x3_launch(n, rest, kb, -1.0f, d_B + k0, ldb,
                                          d_A + static_cast<int64_t>(k0) * lda + k0 + kb, lda, 1.0f, d_B + k0 + kb, ldb,
                                          d_workspace, ws_bytes, s, first);
        } else {
            if (unit) trsm_right_upper_block<true><<<solve_grid(m), 256, 0, s>>>(d_A, lda, d_B, ldb, k0, kb, m);
            else trsm_right_upper_block<false><<<solve_grid(m), 256, 0, s>>>(d_A, lda, d_B, ldb, k0, kb, m);
            PMB_CUDA_TRY(cudaGetLastError());
            if (rest == 0) break;
            // B[:, k1:] -= X_k U[k, k1:] (column-major) == row-major C^T -= U^T X_k^T: M = rest, N = m, K = kb
            st = pmb::sgemm_bf16x3_launch(rest, m, kb, -1.0f, d_A + static_cast<int64_t>(k0 + kb) * lda + k0, lda,
                                          d_B + static_cast<int64_t>(k0) * ldb, ldb, 1.0f,
                                          d_B + static_cast<int64_t>(k0 + kb) * ldb, ldb, d_workspace, ws_bytes, s,
                                          first);
        }
        if (st != PMB_SUCCESS) return st;
        first = false;
    }
    return PMB_SUCCESS;
}
