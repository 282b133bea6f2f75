// Device helpers of the served mixed-size workload driver (served_mix.cpp):
// building an LU task's diagonally dominant input from the shared random pool
// inside the task's GPU callback, and the FP64 error checks that run after the
// timed stream.  The product kernels (tcgen05 GEMM, blocked LU) live in
// libpmb.so; nothing here is on their path.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

// out (n x n, column-major, ld n) = pool block (ld ldp) + diag * I.
__global__ void prepare_lu_kernel(const float* __restrict__ pool, int64_t ldp, float* __restrict__ out, int n,
                                  float diag) {
    const int64_t total = static_cast<int64_t>(n) * n;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t c = e / n, r = e - c * n;
        float v = pool[c * ldp + r];
        if (r == c) v += diag;
        out[e] = v;
    }
}

// sums[0] += sum (C - A*B)^2, sums[1] += sum (A*B)^2, with A*B in FP64.
// Row-major n x n operands; 32 x 32 output tile per 256-thread CTA.
__global__ void __launch_bounds__(256)
gemm_err_kernel(const float* __restrict__ A, int64_t lda, const float* __restrict__ B, int64_t ldb,
                const float* __restrict__ C, int64_t ldc, int n, double* __restrict__ sums) {
    __shared__ double sa[32][33];
    __shared__ double sb[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 row groups
    const int col = blockIdx.x * 32 + tx;
    const int row0 = blockIdx.y * 32;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k0 = 0; k0 < n; k0 += 32) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = ty + 8 * i;
            const int ar = row0 + r, ac = k0 + tx;
            sa[r][tx] = (ar < n && ac < n) ? static_cast<double>(A[static_cast<int64_t>(ar) * lda + ac]) : 0.0;
            const int br = k0 + r;
            sb[r][tx] = (br < n && col < n) ? static_cast<double>(B[static_cast<int64_t>(br) * ldb + col]) : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < 32; ++k) {
            const double b = sb[k][tx];
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[i] = fma(sa[ty + 8 * i][k], b, acc[i]);
        }
        __syncthreads();
    }
    double e2 = 0.0, r2 = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = row0 + ty + 8 * i;
        if (r < n && col < n) {
            const double d = static_cast<double>(C[static_cast<int64_t>(r) * ldc + col]) - acc[i];
            e2 += d * d;
            r2 += acc[i] * acc[i];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        e2 += __shfl_xor_sync(0xffffffffu, e2, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], e2);
        atomicAdd(&sums[1], r2);
    }
}

}  // namespace

extern "C" int sm_prepare_lu(const float* pool, int64_t ldp, float* out, int n, float diag, void* stream) {
    if (n <= 0) return 0;
    prepare_lu_kernel<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(pool, ldp, out, n, diag);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Relative Frobenius error of a row-major fp32 product C against A*B in FP64.
// Synchronous; returns a negative value on a CUDA error.
extern "C" double sm_gemm_rel_error(const float* dA, int64_t lda, const float* dB, int64_t ldb, const float* dC,
                                    int64_t ldc, int n) {
    double* sums = nullptr;
    if (cudaMalloc(&sums, 2 * sizeof(double)) != cudaSuccess) return -1.0;
    cudaMemset(sums, 0, 2 * sizeof(double));
    gemm_err_kernel<<<dim3((n + 31) / 32, (n + 31) / 32), 256>>>(dA, lda, dB, ldb, dC, ldc, n, sums);
    double h[2] = {0.0, 0.0};
    const cudaError_t e = cudaMemcpy(h, sums, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(sums);
    if (e != cudaSuccess) return -1.0;
    return h[1] > 0 ? sqrt(h[0] / h[1]) : sqrt(h[0]);
}
