// Shared helpers of libpmb.so: error reporting through the C ABI, CUDA status
// translation, and small device utilities used by several kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "pmb_capi.h"

namespace pmb {

// Record a printf-style message as the calling thread's last error and return
// `status` (so call sites can `return fail(PMB_INVALID_INDEX, "...")`).
int fail(int status, const char* fmt, ...);

// Translate a CUDA error into PMB_GRAPHICS_CARD_ERROR with a message naming
// the call that failed.
int cuda_fail(cudaError_t err, const char* what);

// Clear the calling thread's last error.
void clear_error();

// Tensor-memory exclusivity of a kernel that allocates TMEM: its CTAs take
// more than half of an SM's shared memory, so no two TMEM-allocating CTAs of
// this library (each of which satisfies the same) are ever resident on one
// SM together.  Two TMEM-allocating CTAs on one SM could wait
// on each other's columns -- for CTA pairs (cta_group::2) even across two
// SMs -- so every TMEM-allocating launch checks this once and fails with
// PMB_BEYOND_LIMITS otherwise.
int tmem_exclusive(const void* kernel, int threads, size_t smem_bytes, const char* name);

// cuTensorMapEncodeTiled, looked up once through the runtime's driver entry
// point (null when the driver does not provide it).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn tensor_map_encoder();

}  // namespace pmb

#define PMB_CUDA_TRY(call)                                          \
    do {                                                            \
        cudaError_t pmb_err_ = (call);                              \
        if (pmb_err_ != cudaSuccess) return pmb::cuda_fail(pmb_err_, #call); \
    } while (0)

#define PMB_CHECK_ARG(cond, ...)                                    \
    do {                                                            \
        if (!(cond)) return pmb::fail(PMB_INVALID_INDEX, __VA_ARGS__); \
    } while (0)

namespace pmb {

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

}  // namespace pmb
