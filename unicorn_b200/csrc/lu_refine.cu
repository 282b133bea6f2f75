// FP64 residual-driven refinement of a solve with the fp32 LU factors.
//
// The reference factors in fp32 and stops there (luDecomposition.cpp:116-125,
// 425-470); this adds the mixed-precision step that recovers FP64 accuracy
// from those factors for a right-hand side b:
//   x_0 = U^-1 L^-1 b
//   repeat: r = b - A x (FP64 sums of the fp32 entries of A), d = U^-1 L^-1 r,
//           x += d
// with L (diagonal included) and U (unit diagonal) read from the packed
// fp32 factorization pmb_lu_decompose produces, and every triangular solve
// carried out in FP64.  After each solve the normwise backward error
// ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) is recorded on the device.
//
// Kernels: the triangular solves run in one 1024-thread CTA each, 32-row
// diagonal blocks solved by one warp with shuffles and the rows below (or
// above) updated by all threads reading the factor columns coalesced; the
// residual is row-parallel over column chunks with FP64 atomic adds.
#include "pmb_common.cuh"

namespace {

constexpr int kTb = 32;          // diagonal block of the triangular solves
constexpr int kSolveThreads = 1024;
constexpr int kResidCols = 64;   // columns per residual CTA

__device__ __forceinline__ double lu_at(const float* __restrict__ LU, int64_t ld, int r, int c) {
    return static_cast<double>(LU[static_cast<int64_t>(c) * ld + r]);
}

// v <- L^-1 v, L = lower triangle of LU with its diagonal.
__global__ void __launch_bounds__(kSolveThreads)
trsv_lower_kernel(const float* __restrict__ LU, int64_t ld, int n, double* __restrict__ v) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k0 = 0; k0 < n; k0 += kTb) {
        const int kb = min(kTb, n - k0);
        if (warp == 0) {
            double y = lane < kb ? v[k0 + lane] : 0.0;
            for (int i = 0; i < kb; ++i) {
                if (lane == i) y /= lu_at(LU, ld, k0 + i, k0 + i);
                const double yi = __shfl_sync(0xffffffffu, y, i);
                if (lane > i && lane < kb) y -= lu_at(LU, ld, k0 + lane, k0 + i) * yi;
            }
            if (lane < kb) v[k0 + lane] = y;
        }
        __syncthreads();
        for (int r = k0 + kb + tid; r < n; r += kSolveThreads) {
            double s = 0.0;
            for (int c = 0; c < kb; ++c) s += lu_at(LU, ld, r, k0 + c) * v[k0 + c];
            v[r] -= s;
        }
        __syncthreads();
    }
}

// v <- U^-1 v, U = strict upper triangle of LU with a unit diagonal.
__global__ void __launch_bounds__(kSolveThreads)
trsv_upper_unit_kernel(const float* __restrict__ LU, int64_t ld, int n, double* __restrict__ v) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k1 = n; k1 > 0; k1 -= kTb) {
        const int k0 = max(0, k1 - kTb), kb = k1 - k0;
        if (warp == 0) {
            double y = lane < kb ? v[k0 + lane] : 0.0;
            for (int i = kb - 1; i >= 0; --i) {
                const double xi = __shfl_sync(0xffffffffu, y, i);
                if (lane < i) y -= lu_at(LU, ld, k0 + lane, k0 + i) * xi;
            }
            if (lane < kb) v[k0 + lane] = y;
        }
        __syncthreads();
        for (int r = tid; r < k0; r += kSolveThreads) {
            double s = 0.0;
            for (int c = 0; c < kb; ++c) s += lu_at(LU, ld, r, k0 + c) * v[k0 + c];
            v[r] -= s;
        }
        __syncthreads();
    }
}

// r -= A0 x over columns [blockIdx.y * kResidCols, +kResidCols); rowabs (if
// given) += |A0| over the same columns.
__global__ void __launch_bounds__(256)
residual_kernel(const float* __restrict__ A0, int64_t lda, int n, const double* __restrict__ x, double* __restrict__ r,
                double* __restrict__ rowabs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j0 = blockIdx.y * kResidCols, j1 = min(n, j0 + kResidCols);
    if (i >= n) return;
    double s = 0.0, sa = 0.0;
    for (int j = j0; j < j1; ++j) {
        const double a = static_cast<double>(A0[static_cast<int64_t>(j) * lda + i]);
        s += a * x[j];
        sa += fabs(a);
    }
    atomicAdd(&r[i], -s);
    if (rowabs) atomicAdd(&rowabs[i], sa);
}

__global__ void axpy_kernel(int n, const double* __restrict__ d, double* __restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += d[i];
}

// berr = max|r| / (max rowabs * max|x| + max|b|), one CTA.
__global__ void __launch_bounds__(1024)
backward_error_kernel(int n, const double* __restrict__ r, const double* __restrict__ x, const double* __restrict__ b,
                      const double* __restrict__ rowabs, double* __restrict__ berr) {
    __shared__ double s[4][32];
    double mr = 0, mx = 0, mb = 0, ma = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        mr = fmax(mr, fabs(r[i]));
        mx = fmax(mx, fabs(x[i]));
        mb = fmax(mb, fabs(b[i]));
        ma = fmax(ma, rowabs[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
        ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s[0][warp] = mr;
        s[1][warp] = mx;
        s[2][warp] = mb;
        s[3][warp] = ma;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < static_cast<int>(blockDim.x / 32); ++w) {
            mr = fmax(mr, s[0][w]);
            mx = fmax(mx, s[1][w]);
            mb = fmax(mb, s[2][w]);
            ma = fmax(ma, s[3][w]);
        }
        mr = fmax(mr, s[0][0]);
        mx = fmax(mx, s[1][0]);
        mb = fmax(mb, s[2][0]);
        ma = fmax(ma, s[3][0]);
        const double den = ma * mx + mb;
        *berr = den > 0 ? mr / den : 0.0;
    }
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" size_t pmb_lu_refine_workspace_bytes(int n) {
    return n <= 0 ? 256 : 3 * align256(8ull * static_cast<size_t>(n));
}

extern "C" int pmb_lu_solve_refined(const float* d_A0, int64_t lda0, const float* d_LU, int64_t ldlu, int n,
                                    const double* d_b, double* d_x, int iterations, double* d_berr, void* d_workspace,
                                    size_t ws_bytes, void* stream) {
    PMB_CHECK_ARG(n >= 1, "n %d < 1", n);
    PMB_CHECK_ARG(d_A0 && d_LU && d_b && d_x && d_berr && d_workspace, "null pointer");
    PMB_CHECK_ARG(lda0 >= n && ldlu >= n, "leading dimensions too small");
    PMB_CHECK_ARG(iterations >= 0 && iterations <= 64, "iterations %d outside [0,64]", iterations);
    PMB_CHECK_ARG(ws_bytes >= pmb_lu_refine_workspace_bytes(n), "refinement workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* w = static_cast<char*>(d_workspace);
    double* r = reinterpret_cast<double*>(w);
    double* d = reinterpret_cast<double*>(w + align256(8ull * n));
    double* rowabs = reinterpret_cast<double*>(w + 2 * align256(8ull * n));
    const size_t vb = 8ull * static_cast<size_t>(n);
    const dim3 rgrid((n + 255) / 256, (n + kResidCols - 1) / kResidCols);
    PMB_CUDA_TRY(cudaMemsetAsync(d_x, 0, vb, s));
    PMB_CUDA_TRY(cudaMemsetAsync(rowabs, 0, vb, s));
    PMB_CUDA_TRY(cudaMemcpyAsync(d, d_b, vb, cudaMemcpyDeviceToDevice, s));  // first correction solves for b
    for (int it = 0; it <= iterations; ++it) {
        trsv_lower_kernel<<<1, kSolveThreads, 0, s>>>(d_LU, ldlu, n, d);
        trsv_upper_unit_kernel<<<1, kSolveThreads, 0, s>>>(d_LU, ldlu, n, d);
        axpy_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, d, d_x);
        PMB_CUDA_TRY(cudaMemcpyAsync(r, d_b, vb, cudaMemcpyDeviceToDevice, s));
        residual_kernel<<<rgrid, 256, 0, s>>>(d_A0, lda0, n, d_x, r, it == 0 ? rowabs : nullptr);
        backward_error_kernel<<<1, 1024, 0, s>>>(n, r, d_x, d_b, rowabs, d_berr + it);
        PMB_CUDA_TRY(cudaGetLastError());
        if (it < iterations) PMB_CUDA_TRY(cudaMemcpyAsync(d, r, vb, cudaMemcpyDeviceToDevice, s));
    }
    return PMB_SUCCESS;
}
