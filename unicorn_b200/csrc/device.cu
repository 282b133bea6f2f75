// Device layer of the C ABI: the only CUDA runtime calls the pm:: runtime
// (libpmlib.so, plain C++) makes go through these entry points -- device
// selection, memory, streams, events, asynchronous copies, kernel launch for
// apps' subtask_gpu_cuda kernels, and CUDA graph capture.  They replace the
// dlsym'd runtime calls of pmCudaInterface (source/code/src/pmCudaInterface.cu
// :69-146, :156-173, :336-339, :474-550).
#include "pmb_common.cuh"

namespace {
cudaMemcpyKind kind_of(int k) {
    switch (k) {
        case PMB_H2D: return cudaMemcpyHostToDevice;
        case PMB_D2H: return cudaMemcpyDeviceToHost;
        case PMB_D2D: return cudaMemcpyDeviceToDevice;
        default: return cudaMemcpyDefault;
    }
}
}  // namespace

extern "C" int pmb_device_count(int* count) {
    PMB_CHECK_ARG(count, "null pointer");
    const cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
    }
    return PMB_SUCCESS;
}

extern "C" int pmb_set_device(int dev) {
    PMB_CUDA_TRY(cudaSetDevice(dev));
    PMB_CUDA_TRY(cudaFree(nullptr));  // create the primary context now
    return PMB_SUCCESS;
}

extern "C" int pmb_device_properties(int dev, char* name, size_t name_len, int* sm_count, int* cc_major,
                                     int* cc_minor) {
    cudaDeviceProp p;
    PMB_CUDA_TRY(cudaGetDeviceProperties(&p, dev));
    if (name && name_len) {
        size_t i = 0;
        for (; i + 1 < name_len && p.name[i]; ++i) name[i] = p.name[i];
        name[i] = 0;
    }
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (cc_major) *cc_major = p.major;
    if (cc_minor) *cc_minor = p.minor;
    return PMB_SUCCESS;
}

extern "C" int pmb_mem_get_info(size_t* free_bytes, size_t* total_bytes) {
    PMB_CHECK_ARG(free_bytes && total_bytes, "null pointer");
    PMB_CUDA_TRY(cudaMemGetInfo(free_bytes, total_bytes));
    return PMB_SUCCESS;
}

extern "C" int pmb_malloc(void** p, size_t bytes) {
    PMB_CHECK_ARG(p, "null pointer");
    const cudaError_t e = cudaMalloc(p, bytes ? bytes : 1);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        *p = nullptr;
        return pmb::fail(PMB_MEMORY_ERROR, "cudaMalloc of %zu bytes failed: out of device memory", bytes);
    }
    PMB_CUDA_TRY(e);
    return PMB_SUCCESS;
}

extern "C" int pmb_free(void* p) {
    if (p) PMB_CUDA_TRY(cudaFree(p));
    return PMB_SUCCESS;
}

extern "C" int pmb_malloc_async(void** p, size_t bytes, void* stream) {
    PMB_CHECK_ARG(p, "null pointer");
    const cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 1, static_cast<cudaStream_t>(stream));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        *p = nullptr;
        return pmb::fail(PMB_MEMORY_ERROR, "cudaMallocAsync of %zu bytes failed: out of device memory", bytes);
    }
    PMB_CUDA_TRY(e);
    return PMB_SUCCESS;
}

extern "C" int pmb_free_async(void* p, void* stream) {
    if (p) PMB_CUDA_TRY(cudaFreeAsync(p, static_cast<cudaStream_t>(stream)));
    return PMB_SUCCESS;
}

extern "C" int pmb_host_alloc(void** p, size_t bytes) {
    PMB_CHECK_ARG(p, "null pointer");
    const cudaError_t e = cudaHostAlloc(p, bytes ? bytes : 1, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return pmb::fail(PMB_MEMORY_ERROR, "cudaHostAlloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return PMB_SUCCESS;
}

extern "C" int pmb_host_free(void* p) {
    if (p) PMB_CUDA_TRY(cudaFreeHost(p));
    return PMB_SUCCESS;
}

extern "C" int pmb_stream_create(void** s) {
    PMB_CHECK_ARG(s, "null pointer");
    cudaStream_t st;
    PMB_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    *s = st;
    return PMB_SUCCESS;
}

extern "C" int pmb_stream_destroy(void* s) {
    if (s) PMB_CUDA_TRY(cudaStreamDestroy(static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_stream_synchronize(void* s) {
    PMB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_event_create(void** e, int timing) {
    PMB_CHECK_ARG(e, "null pointer");
    cudaEvent_t ev;
    PMB_CUDA_TRY(cudaEventCreateWithFlags(&ev, timing ? cudaEventDefault : cudaEventDisableTiming));
    *e = ev;
    return PMB_SUCCESS;
}

extern "C" int pmb_event_destroy(void* e) {
    if (e) PMB_CUDA_TRY(cudaEventDestroy(static_cast<cudaEvent_t>(e)));
    return PMB_SUCCESS;
}

extern "C" int pmb_event_record(void* e, void* s) {
    PMB_CUDA_TRY(cudaEventRecord(static_cast<cudaEvent_t>(e), static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_event_query(void* e) {
    const cudaError_t r = cudaEventQuery(static_cast<cudaEvent_t>(e));
    if (r == cudaSuccess) return PMB_SUCCESS;
    if (r == cudaErrorNotReady) {
        cudaGetLastError();
        return PMB_STATUS_UNAVAILABLE;
    }
    return pmb::cuda_fail(r, "cudaEventQuery");
}

extern "C" int pmb_event_synchronize(void* e) {
    PMB_CUDA_TRY(cudaEventSynchronize(static_cast<cudaEvent_t>(e)));
    return PMB_SUCCESS;
}

extern "C" int pmb_event_elapsed_ms(void* start, void* end, float* ms) {
    PMB_CHECK_ARG(ms, "null pointer");
    PMB_CUDA_TRY(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start), static_cast<cudaEvent_t>(end)));
    return PMB_SUCCESS;
}

extern "C" int pmb_stream_wait_event(void* s, void* e) {
    PMB_CUDA_TRY(cudaStreamWaitEvent(static_cast<cudaStream_t>(s), static_cast<cudaEvent_t>(e), 0));
    return PMB_SUCCESS;
}

extern "C" int pmb_memcpy_async(void* dst, const void* src, size_t bytes, int kind, void* s) {
    if (bytes == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(dst && src, "null pointer");
    PMB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, kind_of(kind), static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_memcpy2d_async(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                                  size_t height, int kind, void* s) {
    if (width == 0 || height == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(dst && src, "null pointer");
    PMB_CUDA_TRY(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, kind_of(kind), static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_memset_async(void* p, int value, size_t bytes, void* s) {
    if (bytes == 0) return PMB_SUCCESS;
    PMB_CUDA_TRY(cudaMemsetAsync(p, value, bytes, static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_launch_kernel(const void* fn, unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by,
                                 unsigned bz, unsigned smem, void** args, void* s) {
    PMB_CHECK_ARG(fn, "null kernel");
    PMB_CUDA_TRY(cudaLaunchKernel(fn, dim3(gx, gy, gz), dim3(bx, by, bz), args, smem, static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_device_synchronize(void) {
    PMB_CUDA_TRY(cudaDeviceSynchronize());
    return PMB_SUCCESS;
}

extern "C" int pmb_graph_begin_capture(void* s) {
    PMB_CUDA_TRY(cudaStreamBeginCapture(static_cast<cudaStream_t>(s), cudaStreamCaptureModeThreadLocal));
    return PMB_SUCCESS;
}

extern "C" int pmb_graph_end_capture(void* s, void** exec) {
    PMB_CHECK_ARG(exec, "null pointer");
    cudaGraph_t g;
    PMB_CUDA_TRY(cudaStreamEndCapture(static_cast<cudaStream_t>(s), &g));
    cudaGraphExec_t ge;
    const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    PMB_CUDA_TRY(e);
    *exec = ge;
    return PMB_SUCCESS;
}

extern "C" int pmb_graph_launch(void* exec, void* s) {
    PMB_CUDA_TRY(cudaGraphLaunch(static_cast<cudaGraphExec_t>(exec), static_cast<cudaStream_t>(s)));
    return PMB_SUCCESS;
}

extern "C" int pmb_graph_destroy(void* exec) {
    if (exec) PMB_CUDA_TRY(cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(exec)));
    return PMB_SUCCESS;
}

extern "C" int pmb_mempool_retain(int dev) {
    cudaMemPool_t pool;
    PMB_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t threshold = UINT64_MAX;  // keep freed blocks for reuse instead of returning them
    PMB_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    return PMB_SUCCESS;
}

extern "C" int pmb_mempool_reserve(int dev, size_t bytes, size_t* reserved) {
    cudaMemPool_t pool;
    PMB_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t cur = 0;
    PMB_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &cur));
    if (cur < bytes) {
        cudaStream_t s;
        PMB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        // One allocation maps the memory; freeing it at once leaves it in the
        // pool (release threshold: keep everything).  Halve on failure.
        for (size_t want = bytes - cur; want >= (size_t(64) << 20); want /= 2) {
            void* p = nullptr;
            const cudaError_t e = cudaMallocAsync(&p, want, s);
            if (e == cudaSuccess) {
                cudaFreeAsync(p, s);
                break;
            }
            cudaGetLastError();
            if (e != cudaErrorMemoryAllocation) {
                cudaStreamDestroy(s);
                return pmb::cuda_fail(e, "cudaMallocAsync (pool reservation)");
            }
        }
        const cudaError_t e = cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        PMB_CUDA_TRY(e);
        PMB_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &cur));
    }
    if (reserved) *reserved = static_cast<size_t>(cur);
    return PMB_SUCCESS;
}

extern "C" int pmb_mempool_trim(int dev, size_t keep_bytes) {
    cudaMemPool_t pool;
    PMB_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
    PMB_CUDA_TRY(cudaMemPoolTrimTo(pool, keep_bytes));
    return PMB_SUCCESS;
}

extern "C" int pmb_mem_available(int dev, size_t* available) {
    PMB_CHECK_ARG(available, "null pointer");
    size_t fr = 0, tot = 0;
    PMB_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    cudaMemPool_t pool;
    PMB_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t reserved = 0, used = 0;
    PMB_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    PMB_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
    *available = fr + (reserved > used ? static_cast<size_t>(reserved - used) : 0);
    return PMB_SUCCESS;
}

// ---------------------------------------------------------------------------
// Many byte ranges in one launch (the device side of ordered redistribution,
// source/code/src/pmRedistributor.cpp:240-283, which copies range by range):
// CTA k copies range k with 16-byte vector moves where source and
// destination agree modulo 16, byte moves at the ends and otherwise.
namespace {

__global__ void __launch_bounds__(256)
copy_ranges_kernel(char* __restrict__ dst, const char* __restrict__ src, const pmb_copy_range* __restrict__ ranges,
                   int n) {
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const pmb_copy_range r = ranges[k];
        const char* s = src + r.src;
        char* d = dst + r.dst;
        size_t len = r.len;
        if (((reinterpret_cast<uintptr_t>(s) ^ reinterpret_cast<uintptr_t>(d)) & 15) == 0) {
            const size_t head = (16 - (reinterpret_cast<uintptr_t>(s) & 15)) & 15;
            const size_t h = head < len ? head : len;
            if (threadIdx.x < h) d[threadIdx.x] = s[threadIdx.x];
            s += h;
            d += h;
            len -= h;
            const size_t nv = len / 16;
            const uint4* sv = reinterpret_cast<const uint4*>(s);
            uint4* dv = reinterpret_cast<uint4*>(d);
            for (size_t i = threadIdx.x; i < nv; i += blockDim.x) dv[i] = sv[i];
            for (size_t i = nv * 16 + threadIdx.x; i < len; i += blockDim.x) d[i] = s[i];
        } else {
            for (size_t i = threadIdx.x; i < len; i += blockDim.x) d[i] = s[i];
        }
    }
}

}  // namespace

extern "C" int pmb_copy_ranges(void* d_dst, const void* d_src, const pmb_copy_range* d_ranges, int n_ranges,
                               void* stream) {
    if (n_ranges <= 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(d_dst && d_src && d_ranges, "null pointer");
    const int grid = n_ranges < 65535 ? n_ranges : 65535;
    copy_ranges_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<char*>(d_dst), static_cast<const char*>(d_src), d_ranges, n_ranges);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}
