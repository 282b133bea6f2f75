// Library-wide C ABI entry points (version, last error, device check) and the
// error plumbing behind them.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "pmb_common.cuh"

namespace pmb {

static thread_local char t_last_error[1024] = {0};

int fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_last_error, sizeof(t_last_error), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_fail(cudaError_t err, const char* what) {
    return fail(PMB_GRAPHICS_CARD_ERROR, "%s failed: %s (%d)", what, cudaGetErrorString(err),
                static_cast<int>(err));
}

void clear_error() { t_last_error[0] = 0; }

int tmem_exclusive(const void* kernel, int threads, size_t smem_bytes, const char* name) {
    (void)kernel;
    (void)threads;
    int dev = 0, per_sm = 0;
    PMB_CUDA_TRY(cudaGetDevice(&dev));
    PMB_CUDA_TRY(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    if (2 * smem_bytes <= static_cast<size_t>(per_sm))
        return fail(PMB_BEYOND_LIMITS, "%s: %zu bytes of shared memory per CTA would let two CTAs holding tensor "
                    "memory share an SM (%d bytes per SM)", name, smem_bytes, per_sm);
    return PMB_SUCCESS;
}

EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

}  // namespace pmb

extern "C" const char* pmb_last_error(void) { return pmb::t_last_error; }

extern "C" const char* pmb_version(void) { return "1_0_0"; }

extern "C" int pmb_device_supported(int dev) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return prop.major == 10 && prop.minor == 0 ? 1 : 0;
}
