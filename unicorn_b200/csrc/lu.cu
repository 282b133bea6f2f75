// luDecomposition subtask kernels: blocked, unpivoted LU of a column-major
// fp32 matrix, in place, in the reference's Crout form.
//
// Semantics (testSuite/luDecomposition/source/code/src/luDecomposition.cpp:
// 116-125 serialLUDecomposition): for each column i the row to the right of
// the diagonal is scaled by 1/a_ii and the trailing block gets the rank-1
// update -= column(i) x row(i).  L therefore keeps the diagonal (the pivots)
// and U is unit upper triangular; A = L*U.  The reference runs it as three
// task stages per BLOCK_DIM step (luDecomposition.h:70-85): factor the
// diagonal block (luDecompositionCUDA.cu:66-97, 2047 x {1-thread kernel,
// cublasSscal, cublasSger}), solve the row and column panels (cublasStrsm,
// :99-151), update the trailing matrix (cublasSgemm, :153-193).
//
// B200 design, per nb-step (nb <= 64, the default 64):
//  1. one CTA factors the diagonal block in FP64, held in registers (one
//     barrier per column), and writes the factors as fp32 into A11 and in
//     FP64 to the workspace;
//  2. one launch solves both panels in FP64 from those factors -- U12 =
//     L11^-1 A12 by forward substitution (a warp per column) and L21 =
//     A21 U11^-1 by substitution with the unit upper U11 (a warp per row) --
//     and writes them both as fp32 and as the BF16 hi/lo operands of step 3;
//  3. A22 -= L21 * U12 runs on the tensor cores (BF16x3, K = 64) in the
//     short-product GEMM kernel, which streams A22 through shared memory by
//     TMA.  (An A22 that TMA cannot address -- unaligned base or row pitch --
//     takes a split pass and the general GEMM kernel instead.)
// Block sizes above 64 factor in a 512-thread CTA that also inverts both
// triangles (W = L11^-1, V = U11^-1, FP64, written as fp32) and solve the
// panels as BF16x3 GEMMs U12 = W * A12, L21 = A21 * V.
// An FP64 check of each finished L column (inside steps 1 and 2, or a
// separate scan for large blocks) tests that partial pivoting would have
// chosen the diagonal (P = I, as diagonally dominant inputs guarantee);
// if not, the factorization still completes unpivoted (the reference never
// pivots) and the call reports it through the workspace flag word.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>

#include "pmb_common.cuh"

extern "C" size_t pmb_gemm_workspace_bytes(int M, int N, int K);
extern "C" int pmb_sgemm_bf16x3(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B,
                                int64_t ldb, float beta, float* C, int64_t ldc, void* workspace, size_t ws_bytes,
                                void* stream);
namespace pmb {
int sgemm_bf16x3_launch(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                        float beta, float* C, int64_t ldc, void* workspace, size_t ws_bytes, cudaStream_t s,
                        bool clear_error);
int gemm_presplit_launch(int M, int N, int kp, float alpha, const __nv_bfloat16* ah, const __nv_bfloat16* al,
                         const __nv_bfloat16* bh, const __nv_bfloat16* bl, float beta, float* C, int64_t ldc,
                         uint32_t* err, cudaStream_t s, bool dependent);
}
extern "C" int pmb_sgemm_plain(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B,
                               int64_t ldb, float beta, float* C, int64_t ldc, void* stream);

namespace {

constexpr int kMaxNb = 128;

// The block-step kernels are chained by programmatic dependent launch: each
// waits here until the previous grid on the stream is complete and its
// writes are visible (at once when it was launched normally), then lets the
// next kernel's launch begin.
__device__ __forceinline__ void grid_dependency_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launch on s, as a programmatic dependent of the previous kernel when `dependent`.
template <typename... KArgs, typename... Args>
cudaError_t launch_chained(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t s, bool dependent,
                           Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = dependent ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
constexpr uint32_t kFlagPivot = 1;      // partial pivoting would have swapped rows
constexpr uint32_t kFlagZeroPivot = 2;  // a pivot was exactly zero

// Element (ii, js) / (is, jj) of a register tile with a run-time index on one
// side, by a select chain (indexing the array at run time would move it to
// local memory).
template <int R, int C>
__device__ __forceinline__ double pick_in_row(const double (&a)[R][C], int ii, int js) {
    double v = a[ii][0];
#pragma unroll
    for (int jj = 1; jj < C; ++jj) v = jj == js ? a[ii][jj] : v;
    return v;
}
template <int R, int C>
__device__ __forceinline__ double pick_in_col(const double (&a)[R][C], int is, int jj) {
    double v = a[0][jj];
#pragma unroll
    for (int ii = 1; ii < R; ++ii) v = ii == is ? a[ii][jj] : v;
    return v;
}

// Factor the kb x kb diagonal block at A (lda) in FP64 and write W = L^-1,
// V = U^-1 (kb x kb, column-major, ld = kb); kb <= NB.
//
// The block lives in registers for the whole kernel: thread (tx = lane,
// ty = warp) owns rows tx + 32*ii of columns ty + WARPS*jj (16 elements for
// NB = 64 on 256 threads, 32 for NB = 128 on 512), a cyclic layout that keeps
// every thread busy as the active part shrinks.  Blocks smaller than NB are
// padded with the identity, which neither phase changes.  Each elimination
// step publishes one column and one row through double-buffered shared
// vectors, so a step costs one barrier.  The published column is zero outside
// the rows a step updates, so the update of every column a warp owns is one
// unconditional FMA per element (the column-ownership test is warp-uniform);
// only the one column a step retires takes per-lane selects.
//  - factorization (Crout): step i publishes column i (zero at rows <= i) and
//    the unscaled row i; the pivot's owner computes 1/a_ii once.  Trailing
//    elements do a_rc -= a_ri * (a_ic / a_ii); row i itself is scaled by the
//    stored reciprocals after the last step (U unit upper, L keeps pivots).
//  - inverses, both triangles in the same steps: W by right-looking forward
//    substitution (row k of W final at step k: its owner scales it while
//    publishing; X_rj -= L_rk W_kj below it) and V by right-looking back
//    substitution from the last row (Y_rj -= U_rq V_qj above row q).  The
//    entries of L (U) consumed at a step are dead after it, so W (V)
//    overwrites the lower (strict upper) triangle in place.
template <int NB, int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
lu_diag_kernel(float* __restrict__ A, int64_t lda, int kb, float* __restrict__ W, float* __restrict__ V,
               uint32_t* __restrict__ flags) {
    constexpr int WARPS = THREADS / 32;
    constexpr int RI = NB / 32, CJ = NB / WARPS;
    static_assert(RI * CJ * THREADS == NB * NB, "every element owned once");
    __shared__ double s_col[2][NB];
    __shared__ double s_row[2][NB];
    __shared__ double s_ucol[2][NB];
    __shared__ double s_vrow[2][NB];
    __shared__ double s_inv[NB];  // 1 / pivot, by step
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double a[RI][CJ];
#pragma unroll
    for (int jj = 0; jj < CJ; ++jj) {
        const int c = ty + WARPS * jj;
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) {
            const int r = tx + 32 * ii;
            a[ii][jj] = (r < kb && c < kb) ? static_cast<double>(A[static_cast<int64_t>(c) * lda + r])
                                           : (r == c ? 1.0 : 0.0);
        }
    }

    // ---- Crout LU ------------------------------------------------------------
    for (int i = 0; i < kb; ++i) {
        const int buf = i & 1;
        if (ty == i % WARPS) {
#pragma unroll
            for (int ii = 0; ii < RI; ++ii) {
                const int r = tx + 32 * ii;
                const double v = pick_in_row(a, ii, i / WARPS);
                s_col[buf][r] = r > i ? v : 0.0;
                if (r == i) {
                    if (v == 0.0) atomicOr(flags, kFlagZeroPivot);
                    s_inv[i] = v != 0.0 ? 1.0 / v : 0.0;
                }
            }
        }
        if (tx == (i & 31)) {
#pragma unroll
            for (int jj = 0; jj < CJ; ++jj) s_row[buf][ty + WARPS * jj] = pick_in_col(a, i >> 5, jj);
        }
        __syncthreads();
        const double inv = s_inv[i];
        double lc[RI];
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) lc[ii] = s_col[buf][tx + 32 * ii];
#pragma unroll
        for (int jj = 0; jj < CJ; ++jj) {
            const int c = ty + WARPS * jj;
            if (c <= i) continue;
            const double u = s_row[buf][c] * inv;  // same address across the warp: broadcast
#pragma unroll
            for (int ii = 0; ii < RI; ++ii) a[ii][jj] = fma(-lc[ii], u, a[ii][jj]);
        }
    }
    __syncthreads();
    // U = unit upper: scale each row of the strict upper triangle by its pivot's reciprocal.
#pragma unroll
    for (int ii = 0; ii < RI; ++ii) {
        const int r = tx + 32 * ii;
        const double sr = r < kb ? s_inv[r] : 1.0;
#pragma unroll
        for (int jj = 0; jj < CJ; ++jj) {
            const int c = ty + WARPS * jj;
            if (r < c) a[ii][jj] *= sr;
        }
    }
#pragma unroll
    for (int jj = 0; jj < CJ; ++jj) {
        const int c = ty + WARPS * jj;
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) {
            const int r = tx + 32 * ii;
            if (r < kb && c < kb) A[static_cast<int64_t>(c) * lda + r] = static_cast<float>(a[ii][jj]);
        }
    }

    // ---- triangular inverses (FP64), W from the top, V from the bottom -------
    for (int st = 0; st < kb; ++st) {
        const int buf = st & 1;
        const int k = st, q = kb - 1 - st;
        const double dinv = s_inv[k];
        if (tx == (k & 31)) {  // row k: publish X_kj (j < k) and scale it into W_kj in place
#pragma unroll
            for (int jj = 0; jj < CJ; ++jj) {
                const int c = ty + WARPS * jj;
                const double x = pick_in_col(a, k >> 5, jj);
                s_row[buf][c] = c < k ? x : 0.0;
                const bool scale = c < k;
#pragma unroll
                for (int ii = 0; ii < RI; ++ii) a[ii][jj] = (scale && ii == (k >> 5)) ? x * dinv : a[ii][jj];
            }
        }
        if (ty == k % WARPS) {  // column k of L below the diagonal (zero elsewhere)
#pragma unroll
            for (int ii = 0; ii < RI; ++ii) {
                const int r = tx + 32 * ii;
                const double v = pick_in_row(a, ii, k / WARPS);
                s_col[buf][r] = r > k ? v : 0.0;
            }
        }
        if (tx == (q & 31)) {  // row q: Y_qj (j > q)
#pragma unroll
            for (int jj = 0; jj < CJ; ++jj) {
                const int c = ty + WARPS * jj;
                const double y = pick_in_col(a, q >> 5, jj);
                s_vrow[buf][c] = c > q ? y : 0.0;
            }
        }
        if (ty == q % WARPS) {  // column q of U above the diagonal (zero elsewhere)
#pragma unroll
            for (int ii = 0; ii < RI; ++ii) {
                const int r = tx + 32 * ii;
                const double v = pick_in_row(a, ii, q / WARPS);
                s_ucol[buf][r] = r < q ? v : 0.0;
            }
        }
        __syncthreads();
        double lc[RI], uc[RI];
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) {
            lc[ii] = s_col[buf][tx + 32 * ii];
            uc[ii] = s_ucol[buf][tx + 32 * ii];
        }
#pragma unroll
        for (int jj = 0; jj < CJ; ++jj) {
            const int c = ty + WARPS * jj;
            if (c < k) {  // X_rc -= L_rk W_kc for rows below k
                const double w = s_row[buf][c] * dinv;
#pragma unroll
                for (int ii = 0; ii < RI; ++ii) a[ii][jj] = fma(-lc[ii], w, a[ii][jj]);
            } else if (c == k) {  // the retiring column: W_kk and -L_rk W_kk below it
#pragma unroll
                for (int ii = 0; ii < RI; ++ii) {
                    const int r = tx + 32 * ii;
                    a[ii][jj] = r == k ? dinv : (r > k ? -lc[ii] * dinv : a[ii][jj]);
                }
            }
            if (c > q) {  // Y_rc -= U_rq V_qc for rows above q
                const double v = s_vrow[buf][c];
#pragma unroll
                for (int ii = 0; ii < RI; ++ii) a[ii][jj] = fma(-uc[ii], v, a[ii][jj]);
            } else if (c == q) {  // the retiring column: -U_rq above the diagonal
#pragma unroll
                for (int ii = 0; ii < RI; ++ii) {
                    const int r = tx + 32 * ii;
                    a[ii][jj] = r < q ? -uc[ii] : a[ii][jj];
                }
            }
        }
    }
#pragma unroll
    for (int jj = 0; jj < CJ; ++jj) {
        const int c = ty + WARPS * jj;
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) {
            const int r = tx + 32 * ii;
            if (r < kb && c < kb) {
                const int64_t e = static_cast<int64_t>(c) * kb + r;
                W[e] = r >= c ? static_cast<float>(a[ii][jj]) : 0.0f;
                V[e] = r < c ? static_cast<float>(a[ii][jj]) : (r == c ? 1.0f : 0.0f);
            }
        }
    }
}

// The 64 x 64 diagonal block with every step unrolled: Crout factorization in
// FP64, the factors written to A11 (fp32) and, in FP64, to F (64 x 64,
// column-major: L with its diagonal, U's strict upper part) for the panel
// solves.  The block is always factored as 64 x 64 (a smaller block is padded
// with the identity, whose factors are the identity), so every step's owner
// warp, owner lane and register index are compile-time constants -- no select
// chains to reach a register.  Same algorithm and shared-memory protocol as
// the factorization half of lu_diag_kernel: 256 threads, thread (tx, ty) owns
// rows tx, tx + 32 of columns ty + 8*jj.  The in-block part of the pivot check
// (L entries below a pivot inside the block) is done here; lu_panel_kernel
// checks the rows below the block.
__global__ void __launch_bounds__(256, 1)
lu_diag64_kernel(float* __restrict__ A, int64_t lda, int kb, double* __restrict__ F, uint32_t* __restrict__ flags) {
    grid_dependency_wait();
    constexpr int NB = 64, WARPS = 8, RI = 2, CJ = 8;
    __shared__ double s_col[2][NB];
    __shared__ double s_row[2][NB];
    __shared__ double s_inv[NB];
    __shared__ double s_piv[NB];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double a[RI][CJ];
#pragma unroll
    for (int jj = 0; jj < CJ; ++jj) {
        const int c = ty + WARPS * jj;
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) {
            const int r = tx + 32 * ii;
            a[ii][jj] = (r < kb && c < kb) ? static_cast<double>(A[static_cast<int64_t>(c) * lda + r])
                                           : (r == c ? 1.0 : 0.0);
        }
    }

#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int buf = i & 1;
        if (ty == i % WARPS) {
#pragma unroll
            for (int ii = 0; ii < RI; ++ii) {
                const int r = tx + 32 * ii;
                const double v = a[ii][i / WARPS];
                s_col[buf][r] = r > i ? v : 0.0;
                if (r == i) {
                    if (v == 0.0) atomicOr(flags, kFlagZeroPivot);
                    s_inv[i] = v != 0.0 ? 1.0 / v : 0.0;
                    s_piv[i] = v;
                }
            }
        }
        if (tx == (i & 31)) {
#pragma unroll
            for (int jj = 0; jj < CJ; ++jj) s_row[buf][ty + WARPS * jj] = a[i >> 5][jj];
        }
        __syncthreads();
        const double inv = s_inv[i];
        double lc[RI];
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) lc[ii] = s_col[buf][tx + 32 * ii];
#pragma unroll
        for (int jj = 0; jj < CJ; ++jj) {
            if (ty + WARPS * jj <= i) continue;
            const double u = s_row[buf][ty + WARPS * jj] * inv;
#pragma unroll
            for (int ii = 0; ii < RI; ++ii) a[ii][jj] = fma(-lc[ii], u, a[ii][jj]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int ii = 0; ii < RI; ++ii) {
        const int r = tx + 32 * ii;
        const double sr = s_inv[r];
#pragma unroll
        for (int jj = 0; jj < CJ; ++jj)
            if (r < ty + WARPS * jj) a[ii][jj] *= sr;
    }
#pragma unroll
    for (int jj = 0; jj < CJ; ++jj) {
        const int c = ty + WARPS * jj;
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) {
            const int r = tx + 32 * ii;
            if (r < kb && c < kb) A[static_cast<int64_t>(c) * lda + r] = static_cast<float>(a[ii][jj]);
        }
    }

#pragma unroll
    for (int jj = 0; jj < CJ; ++jj) {
        const int c = ty + WARPS * jj;
#pragma unroll
        for (int ii = 0; ii < RI; ++ii) {
            const int r = tx + 32 * ii;
            F[c * NB + r] = a[ii][jj];  // the whole padded block: identity outside kb x kb
            // Partial pivoting would swap rows if an L entry below a pivot were larger.
            if (r > c && c < kb && fabs(a[ii][jj]) > fabs(s_piv[c])) atomicOr(flags, kFlagPivot);
        }
    }
}

// hi/lo bf16 split of two values per lane into a 64-wide operand row.
__device__ __forceinline__ void split_row(__nv_bfloat16* hi, __nv_bfloat16* lo, int64_t base, int lane, float f0,
                                          float f1) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(f0), h1 = __float2bfloat16_rn(f1);
    hi[base + lane] = h0;
    hi[base + lane + 32] = h1;
    lo[base + lane] = __float2bfloat16_rn(f0 - __bfloat162float(h0));
    lo[base + lane + 32] = __float2bfloat16_rn(f1 - __bfloat162float(h1));
}

// Panel solves of one block step from the FP64 factors F of the diagonal
// block (replacing products with explicit inverses):
//   U12 = L11^-1 A12  -- one warp per column of A12 (kb x rest): forward
//                        substitution, lane l holding rows l and l + 32;
//   L21 = A21 U11^-1  -- one warp per row of A21 (rest x kb): U11 unit upper,
//                        lane l holding columns l and l + 32.
// Blocks [0, col_blocks) take columns and need only L11; the others take rows
// and need only U11, so each block stages one 64 x 64 factor in shared memory
// (L column-major, U transposed: the lanes' reads of a step are consecutive).
// Each step broadcasts the finished unknown with a shuffle.  Rows of L21 also
// finish the pivot check: an entry larger than its column's pivot means
// partial pivoting would have swapped rows.  T = double on the split-precision
// path, float for the plain FP32 form.  Launched with 256 threads.
//
// With uh non-null the kernel also writes the trailing update's operands in
// the GEMM's split form (hi = bf16(x), lo = bf16(x - hi) of the stored fp32 x,
// K-major, 64 wide, zero beyond kb): uh/ul row m = U12 column m, lh/ll row r =
// L21 row r -- what a split pass over the fp32 panels would produce.
template <typename T>
__global__ void __launch_bounds__(256)
lu_panel_kernel(float* __restrict__ A, int64_t lda, int k0, int kb, int rest, int col_blocks,
                const double* __restrict__ F, uint32_t* __restrict__ flags, __nv_bfloat16* __restrict__ uh,
                __nv_bfloat16* __restrict__ ul, __nv_bfloat16* __restrict__ lh, __nv_bfloat16* __restrict__ ll) {
    grid_dependency_wait();
    constexpr int NB = 64;
    __shared__ T sF[NB * NB];
    __shared__ T sDiag[NB];
    const bool cols = blockIdx.x < col_blocks;
#pragma unroll
    for (int k = 0; k < NB * NB / 256; ++k) {  // 16 independent loads in flight per thread
        // Consecutive threads write consecutive shared words (no bank conflicts);
        // the row blocks read F transposed for that (strided, from L2).
        const int e = threadIdx.x + 256 * k;
        const int hi = e / NB, lo = e - hi * NB;
        const int c = cols ? hi : lo, r = cols ? lo : hi;
        const double f = F[c * NB + r];
        sF[e] = cols ? (r >= c ? static_cast<T>(f) : T(0))    // sF[c * 64 + r] = L_rc
                     : (r < c ? static_cast<T>(f) : T(0));    // sF[r * 64 + c] = U_rc
        if (r == c) sDiag[r] = cols ? T(1) / static_cast<T>(f) : static_cast<T>(fabs(f));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    constexpr int wpb = 256 / 32;
    if (cols) {
        for (int item = blockIdx.x * wpb + (threadIdx.x >> 5); item < rest; item += col_blocks * wpb) {
            float* col = A + static_cast<int64_t>(k0 + kb + item) * lda + k0;  // rows k0.. of column k0+kb+item
            T x0 = lane < kb ? static_cast<T>(col[lane]) : T(0);
            T x1 = lane + 32 < kb ? static_cast<T>(col[lane + 32]) : T(0);
#pragma unroll 8
            for (int i = 0; i < NB; ++i) {
                const T xi = __shfl_sync(0xffffffffu, i < 32 ? x0 : x1, i & 31) * sDiag[i];
                if (lane == (i & 31)) {
                    if (i < 32) x0 = xi; else x1 = xi;
                }
                if (lane > i) x0 -= sF[i * NB + lane] * xi;
                if (lane + 32 > i) x1 -= sF[i * NB + lane + 32] * xi;
            }
            const float f0 = static_cast<float>(x0), f1 = static_cast<float>(x1);
            if (lane < kb) col[lane] = f0;
            if (lane + 32 < kb) col[lane + 32] = f1;
            if (uh) split_row(uh, ul, static_cast<int64_t>(item) * NB, lane, f0, f1);
        }
    } else {
        const int row_blocks = gridDim.x - col_blocks;
        for (int item = (blockIdx.x - col_blocks) * wpb + (threadIdx.x >> 5); item < rest; item += row_blocks * wpb) {
            float* row = A + static_cast<int64_t>(k0) * lda + k0 + kb + item;  // columns k0.. of row k0+kb+item
            T x0 = lane < kb ? static_cast<T>(row[static_cast<int64_t>(lane) * lda]) : T(0);
            T x1 = lane + 32 < kb ? static_cast<T>(row[static_cast<int64_t>(lane + 32) * lda]) : T(0);
#pragma unroll 8
            for (int c = 0; c < NB; ++c) {
                const T xc = __shfl_sync(0xffffffffu, c < 32 ? x0 : x1, c & 31);
                if (lane > c) x0 -= xc * sF[c * NB + lane];
                if (lane + 32 > c) x1 -= xc * sF[c * NB + lane + 32];
            }
            bool bigger = false;
            const float f0 = static_cast<float>(x0), f1 = static_cast<float>(x1);
            if (lane < kb) {
                row[static_cast<int64_t>(lane) * lda] = f0;
                bigger |= fabs(x0) > sDiag[lane];
            }
            if (lane + 32 < kb) {
                row[static_cast<int64_t>(lane + 32) * lda] = f1;
                bigger |= fabs(x1) > sDiag[lane + 32];
            }
            if (uh) split_row(lh, ll, static_cast<int64_t>(item) * NB, lane, f0, f1);
            if (__any_sync(0xffffffffu, bigger) && lane == 0) atomicOr(flags, kFlagPivot);
        }
    }
}

// FP64 pivot check of finished L columns k0..k0+kb-1 (rows k0+i..n-1): would
// partial pivoting keep the diagonal?  One warp per column.
__global__ void lu_pivot_check_kernel(const float* __restrict__ A, int64_t lda, int n, int k0, int kb,
                                      uint32_t* __restrict__ flags) {
    const int col = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (col >= kb) return;
    const int j = k0 + col;
    const float* cp = A + static_cast<int64_t>(j) * lda;
    const double d = fabs(static_cast<double>(cp[j]));
    double mx = 0.0;
    for (int r = j + 1 + lane; r < n; r += 32) mx = fmax(mx, fabs(static_cast<double>(cp[r])));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0 && mx > d) atomicOr(flags, kFlagPivot);
}

// Column-major copy of an r x c block (both with their leading dimensions).
__global__ void copy_block_kernel(const float* __restrict__ src, int64_t lds, float* __restrict__ dst, int64_t ldd,
                                  int rows, int cols) {
    const int64_t total = static_cast<int64_t>(rows) * cols;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t c = e / rows, r = e - c * rows;
        dst[c * ldd + r] = src[c * lds + r];
    }
}

// ||A - L*U||_F^2 and ||A||_F^2 in FP64 (L lower with diagonal, U unit upper,
// both read from the packed LU).  16 x 16 output tiles, one per CTA.
__global__ void lu_residual_kernel(const float* __restrict__ A0, int64_t lda0, const float* __restrict__ LU,
                                   int64_t ldl, int n, double* __restrict__ sums) {
    __shared__ double Ls[16][17];
    __shared__ double Us[16][17];
    const int tr = threadIdx.x % 16, tc = threadIdx.x / 16;
    const int r = blockIdx.y * 16 + tr, c = blockIdx.x * 16 + tc;
    double acc = 0.0;
    for (int p0 = 0; p0 < n; p0 += 16) {
        {
            const int p = p0 + tc;  // L[r][p]
            double l = 0.0;
            if (r < n && p < n && p <= r) l = LU[static_cast<int64_t>(p) * ldl + r];
            Ls[tr][tc] = l;
            const int q = p0 + tr;  // U[q][c]
            double u = 0.0;
            if (q < n && c < n) u = q < c ? static_cast<double>(LU[static_cast<int64_t>(c) * ldl + q]) : (q == c ? 1.0 : 0.0);
            Us[tr][tc] = u;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) acc += Ls[tr][k] * Us[k][tc];
        __syncthreads();
    }
    double d2 = 0.0, a2 = 0.0;
    if (r < n && c < n) {
        const double a = A0[static_cast<int64_t>(c) * lda0 + r];
        d2 = (a - acc) * (a - acc);
        a2 = a * a;
    }
    for (int o = 16; o > 0; o >>= 1) {
        d2 += __shfl_xor_sync(0xffffffffu, d2, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], d2);
        atomicAdd(&sums[1], a2);
    }
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

constexpr int kPanelNb = 64;  // block sizes up to this use the FP64 factor + panel-solve path

struct LuWs {
    uint32_t* flags;
    double* F;  // FP64 factors of the diagonal block (kPanelNb x kPanelNb)
    __nv_bfloat16 *uh, *ul, *lh, *ll;  // split trailing-update operands, n x kPanelNb each
    float* W;
    float* V;
    float* panel;
    void* gemm;
    size_t gemm_bytes;
};

LuWs carve(void* ws, int n, int nb) {
    char* p = static_cast<char*>(ws);
    LuWs w;
    w.flags = reinterpret_cast<uint32_t*>(p);  // word 1 = flags (pmb_scratch_error)
    p += 256;
    w.F = reinterpret_cast<double*>(p);
    p += align256(static_cast<size_t>(kPanelNb) * kPanelNb * 8);
    __nv_bfloat16** split[4] = {&w.uh, &w.ul, &w.lh, &w.ll};
    for (auto* b : split) {
        *b = reinterpret_cast<__nv_bfloat16*>(p);
        p += align256(static_cast<size_t>(n) * kPanelNb * 2);
    }
    w.W = reinterpret_cast<float*>(p);
    p += align256(static_cast<size_t>(nb) * nb * 4);
    w.V = reinterpret_cast<float*>(p);
    p += align256(static_cast<size_t>(nb) * nb * 4);
    w.panel = reinterpret_cast<float*>(p);
    p += align256(static_cast<size_t>(nb) * n * 4);
    w.gemm = p;
    w.gemm_bytes = pmb_gemm_workspace_bytes(n, n, nb);
    return w;
}

// Look-ahead: per caller stream (and device) a high-priority stream that runs
// the serial chain -- diagonal block, panel solves, the next block column of
// the update -- while the rest of each trailing update runs on the caller's
// stream, so the block scheduler hands the chain's small grids the next free
// SM ahead of the update's tiles.  Reusable events order them (chain ready ->
// rest of the update may start; rest done -> next panel may start; start and
// end hand-offs with the caller's stream); each wait is enqueued before its
// event is recorded again, so one set of events serves every step.
struct SideStream {
    cudaStream_t hi = nullptr;
    cudaEvent_t panel_done = nullptr, rest_done = nullptr, start = nullptr, end = nullptr;
};

bool side_stream_for(cudaStream_t s, SideStream& out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    static std::mutex mu;
    static std::map<std::pair<int, cudaStream_t>, SideStream> sides;
    std::lock_guard<std::mutex> g(mu);
    auto it = sides.find({dev, s});
    if (it != sides.end()) {
        out = it->second;
        return true;
    }
    SideStream ss;
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ss.hi, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&ss.panel_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ss.rest_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ss.start, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ss.end, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    sides[{dev, s}] = ss;
    out = ss;
    return true;
}

}  // namespace

extern "C" size_t pmb_lu_workspace_bytes(int n, int nb) {
    if (n <= 0 || nb <= 0) return 256;
    return 256 + align256(static_cast<size_t>(kPanelNb) * kPanelNb * 8) +
           4 * align256(static_cast<size_t>(n) * kPanelNb * 2) + 2 * align256(static_cast<size_t>(nb) * nb * 4) + align256(static_cast<size_t>(nb) * n * 4) +
           pmb_gemm_workspace_bytes(n, n, nb);
}

// Blocked LU.  Block sizes up to 64 take three launches a step: the FP64
// diagonal factorization (with the in-block pivot check), the panel solves
// (U12, L21 and the rest of the pivot check) and the trailing update
// A22 -= L21 U12.  With look-ahead (block sizes up to 64, tcgen05 path, the
// stream not being captured, PMB_LU_LOOKAHEAD not 0) the update is split: the
// next block column first, on the high-priority chain stream, so the next
// diagonal block can start; the rest on the caller's stream, overlapping that
// diagonal factorization, and the next panel solve waits for it.  Larger blocks form explicit inverses W = L11^-1 and
// V = U11^-1 and solve the panels as products.  `plain` selects FP32 solves
// and the FP32 SIMT GEMM (the one-task-at-a-time baseline) instead of FP64
// solves and the tcgen05 BF16x3 GEMM.
static int lu_impl(float* A, int n, int64_t lda, int nb, void* workspace, size_t ws_bytes, cudaStream_t s,
                   bool plain) {
    PMB_CHECK_ARG(n >= 0, "negative size");
    if (n == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(A && workspace, "null pointer");
    PMB_CHECK_ARG(lda >= n, "lda %lld < n %d", (long long)lda, n);
    PMB_CHECK_ARG(nb >= 1 && nb <= kMaxNb, "block size %d outside [1,%d]", nb, kMaxNb);
    PMB_CHECK_ARG((reinterpret_cast<uintptr_t>(workspace) & 255) == 0, "workspace must be 256-byte aligned");
    PMB_CHECK_ARG(ws_bytes >= pmb_lu_workspace_bytes(n, nb), "LU workspace too small");
    LuWs w = carve(workspace, n, nb);
    PMB_CUDA_TRY(cudaMemsetAsync(workspace, 0, 256, s));
    if (!plain) PMB_CUDA_TRY(cudaMemsetAsync(w.gemm, 0, 256, s));  // the products' error word, cleared once
    static const bool lookahead_on = [] {
        const char* v = getenv("PMB_LU_LOOKAHEAD");
        return !(v && v[0] == '0');
    }();
    SideStream side;
    bool lookahead = false;
    if (lookahead_on && !plain && nb <= kPanelNb) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone)
            lookahead = side_stream_for(s, side);
        cudaGetLastError();
    }
    bool rest_pending = false;  // the caller's stream holds the rest of the previous update
    cudaStream_t const caller = s;
    if (lookahead) {
        // The chain starts after everything before it on the caller's stream.
        PMB_CUDA_TRY(cudaEventRecord(side.start, caller));
        PMB_CUDA_TRY(cudaStreamWaitEvent(side.hi, side.start, 0));
        s = side.hi;
    }
    for (int k0 = 0; k0 < n; k0 += nb) {
        const int kb = n - k0 < nb ? n - k0 : nb;
        const int rest = n - k0 - kb;
        float* A11 = A + static_cast<int64_t>(k0) * lda + k0;
        float* A12 = A + static_cast<int64_t>(k0 + kb) * lda + k0;  // kb x rest
        float* A21 = A + static_cast<int64_t>(k0) * lda + k0 + kb;  // rest x kb
        float* A22 = A + static_cast<int64_t>(k0 + kb) * lda + k0 + kb;
        int st;
        if (nb <= kPanelNb) {
            // The first diagonal block waits for all earlier work on the stream;
            // later ones follow the previous step's update as dependents.
            PMB_CUDA_TRY(launch_chained(lu_diag64_kernel, 1, 256, s, k0 > 0, A11, lda, kb, w.F, &w.flags[1]));
            if (rest == 0) continue;
            const int half = std::min((rest + 7) / 8, 4 * 148);  // blocks per side, 8 warps (items) each
            if (rest_pending) {
                // The panel solve reads what the rest of the previous update writes,
                // and overwrites the split operands that update reads.
                PMB_CUDA_TRY(cudaStreamWaitEvent(s, side.rest_done, 0));
                rest_pending = false;
            }
            if (plain) {
                PMB_CUDA_TRY(launch_chained(lu_panel_kernel<float>, 2 * half, 256, s, true, A, lda, k0, kb, rest, half,
                                            w.F, &w.flags[1], static_cast<__nv_bfloat16*>(nullptr),
                                            static_cast<__nv_bfloat16*>(nullptr), static_cast<__nv_bfloat16*>(nullptr),
                                            static_cast<__nv_bfloat16*>(nullptr)));
            } else {
                // The update reads and writes A22 by TMA when it is 16-byte aligned with a
                // row pitch that is a multiple of 16 bytes; the panel kernel then hands it
                // the split operands directly.
                const bool direct = (reinterpret_cast<uintptr_t>(A22) & 15) == 0 && (lda & 3) == 0;
                PMB_CUDA_TRY(launch_chained(lu_panel_kernel<double>, 2 * half, 256, s, true, A, lda, k0, kb, rest,
                                            half, w.F, &w.flags[1], direct ? w.uh : nullptr, w.ul, w.lh, w.ll));
                if (direct) {
                    // A22 -= L21 * U12 == row-major (U12^T)(L21^T); a timed-out wait shows as flag 4.
                    // Row-major rows of C are columns of A22; rows of the U12^T operand
                    // are kPanelNb split elements apart.
                    const int kn = lookahead ? std::min(nb, rest) : rest;
                    if (kn < rest) {
                        PMB_CUDA_TRY(cudaEventRecord(side.panel_done, s));
                        PMB_CUDA_TRY(cudaStreamWaitEvent(caller, side.panel_done, 0));
                        const size_t off = static_cast<size_t>(kn) * kPanelNb;
                        st = pmb::gemm_presplit_launch(rest - kn, rest, kPanelNb, -1.0f, w.uh + off, w.ul + off, w.lh,
                                                       w.ll, 1.0f, A22 + static_cast<int64_t>(kn) * lda, lda,
                                                       &w.flags[1], caller, false);
                        if (st != PMB_SUCCESS) return st;
                        PMB_CUDA_TRY(cudaEventRecord(side.rest_done, caller));
                        rest_pending = true;
                    }
                    st = pmb::gemm_presplit_launch(kn, rest, kPanelNb, -1.0f, w.uh, w.ul, w.lh, w.ll, 1.0f, A22, lda,
                                                   &w.flags[1], s, true);
                    if (st != PMB_SUCCESS) return st;
                    continue;
                }
            }
        } else {
            lu_diag_kernel<128, 512><<<1, 512, 0, s>>>(A11, lda, kb, w.W, w.V, &w.flags[1]);
            PMB_CUDA_TRY(cudaGetLastError());
            if (rest > 0) {
                if (plain) {
                    // The SIMT kernel reads its operands in place: solve into the panel buffer, copy back.
                    st = pmb_sgemm_plain(rest, kb, kb, 1.0f, A12, lda, w.W, kb, 0.0f, w.panel, kb, s);
                    if (st != PMB_SUCCESS) return st;
                    copy_block_kernel<<<296, 256, 0, s>>>(w.panel, kb, A12, lda, kb, rest);
                    PMB_CUDA_TRY(cudaGetLastError());
                    st = pmb_sgemm_plain(kb, rest, kb, 1.0f, w.V, kb, A21, lda, 0.0f, w.panel, rest, s);
                    if (st != PMB_SUCCESS) return st;
                    copy_block_kernel<<<296, 256, 0, s>>>(w.panel, rest, A21, lda, rest, kb);
                    PMB_CUDA_TRY(cudaGetLastError());
                } else {
                    // The split pass copies the operands first, so each panel solve writes
                    // over its own operand: two launches per product, no copy back.
                    // U12 = W * A12 (column-major) == row-major (A12^T)(W^T): M = rest, N = kb, K = kb
                    st = pmb::sgemm_bf16x3_launch(rest, kb, kb, 1.0f, A12, lda, w.W, kb, 0.0f, A12, lda, w.gemm,
                                                  w.gemm_bytes, s, false);
                    if (st != PMB_SUCCESS) return st;
                    // L21 = A21 * V (column-major) == row-major (V^T)(A21^T): M = kb, N = rest, K = kb
                    st = pmb::sgemm_bf16x3_launch(kb, rest, kb, 1.0f, w.V, kb, A21, lda, 0.0f, A21, lda, w.gemm,
                                                  w.gemm_bytes, s, false);
                    if (st != PMB_SUCCESS) return st;
                }
            }
            lu_pivot_check_kernel<<<(kb + 7) / 8, 256, 0, s>>>(A, lda, n, k0, kb, &w.flags[1]);
            PMB_CUDA_TRY(cudaGetLastError());
            if (rest == 0) continue;
        }
        // A22 -= L21 * U12 (column-major) == row-major (U12^T)(L21^T): M = rest, N = rest, K = kb
        if (plain) st = pmb_sgemm_plain(rest, rest, kb, -1.0f, A12, lda, A21, lda, 1.0f, A22, lda, s);
        else st = pmb::sgemm_bf16x3_launch(rest, rest, kb, -1.0f, A12, lda, A21, lda, 1.0f, A22, lda, w.gemm,
                                           w.gemm_bytes, s, false);
        if (st != PMB_SUCCESS) return st;
    }
    // The caller's stream completes only after the chain's last kernel.
    if (lookahead) {
        PMB_CUDA_TRY(cudaEventRecord(side.end, s));
        PMB_CUDA_TRY(cudaStreamWaitEvent(caller, side.end, 0));
    }
    return PMB_SUCCESS;
}

extern "C" int pmb_lu_decompose(float* d_A, int n, int64_t lda, int nb, void* d_workspace, size_t ws_bytes,
                                void* stream) {
    return lu_impl(d_A, n, lda, nb, d_workspace, ws_bytes, static_cast<cudaStream_t>(stream), false);
}

extern "C" int pmb_lu_decompose_plain(float* d_A, int n, int64_t lda, int nb, void* d_workspace, size_t ws_bytes,
                                      void* stream) {
    return lu_impl(d_A, n, lda, nb, d_workspace, ws_bytes, static_cast<cudaStream_t>(stream), true);
}

extern "C" int pmb_lu_residual_f64(const float* d_A0, int64_t lda0, const float* d_LU, int64_t ldlu, int n,
                                   double* d_sums, void* stream) {
    PMB_CHECK_ARG(d_A0 && d_LU && d_sums && n >= 1, "bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    PMB_CUDA_TRY(cudaMemsetAsync(d_sums, 0, 2 * sizeof(double), s));
    lu_residual_kernel<<<dim3((n + 15) / 16, (n + 15) / 16), 256, 0, s>>>(d_A0, lda0, d_LU, ldlu, n, d_sums);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}
