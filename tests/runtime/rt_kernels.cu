// App-style subtask_gpu_cuda kernel used by the runtime self-test: the
// runtime launches it with (pmTaskInfo, pmDeviceInfo*, pmSubtaskInfo,
// pmStatus*) by value, exactly as an unchanged app kernel is launched.
#include "pmPublicDefinitions.h"

using namespace pm;

struct RtConf {
    int add;     // constant added to every element
    int ld;      // row pitch of the whole matrix, in ints (NATURAL views)
};

// Per-subtask scratch (PRE_SUBTASK_TO_SUBTASK): {extra, rows, cols}.
// out[r][c] = in[r][c] + add + extra, staged through reserved device memory.
__global__ void rt_add_kernel(pmTaskInfo ti, pmDeviceInfo* di, pmSubtaskInfo si, pmStatus* st) {
    const RtConf* conf = static_cast<const RtConf*>(ti.taskConf);
    const int* in = static_cast<const int*>(si.memInfo[0].ptr);
    int* out = static_cast<int*>(si.memInfo[1].ptr);
    const int* scratch = static_cast<const int*>(si.gpuContext.scratchBuffer);
    const int extra = scratch[0], rows = scratch[1], cols = scratch[2];
    const int in_ld = si.memInfo[0].visibilityType == SUBSCRIPTION_NATURAL ? conf->ld : cols;
    const int out_ld = si.memInfo[1].visibilityType == SUBSCRIPTION_NATURAL ? conf->ld : cols;
    int* reserved = static_cast<int*>(si.gpuContext.reservedGlobalMem);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < rows * cols; e += gridDim.x * blockDim.x) {
        const int r = e / cols, c = e % cols;
        int v = in[r * in_ld + c] + conf->add + extra;
        if (reserved) {
            reserved[e] = v;
            v = reserved[e];
        }
        out[r * out_ld + c] = v;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && di->deviceType != GPU_CUDA) *st = pmFatalError;
}

extern "C" void* rt_add_kernel_ptr() { return reinterpret_cast<void*>(&rt_add_kernel); }

// Reduction self-test: subtask s reads row s of an N x words input and writes
// its copy of the output range, out[j] = in[j] (copy) or out[j] += in[j]
// (accumulate, int32: the copy starts from the address space's bytes).
struct RtRowConf {
    int words;       // 32-bit words per row
    int accumulate;  // 0: copy, 1: add to the subscribed output
    int type, op;    // reduction data type and operation
};

__global__ void rt_row_kernel(pmTaskInfo ti, pmDeviceInfo* di, pmSubtaskInfo si, pmStatus* st) {
    const RtRowConf* conf = static_cast<const RtRowConf*>(ti.taskConf);
    const unsigned* in = static_cast<const unsigned*>(si.memInfo[0].ptr);
    unsigned* out = static_cast<unsigned*>(si.memInfo[1].ptr);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < conf->words; j += gridDim.x * blockDim.x)
        out[j] = conf->accumulate ? out[j] + in[j] : in[j];
}

extern "C" void* rt_row_kernel_ptr() { return reinterpret_cast<void*>(&rt_row_kernel); }

// Redistribution self-test: subtask s groups its chunk of int keys by bucket
// (key mod buckets, stable) into its output chunk and leaves the bucket sizes
// in its SUBTASK_TO_POST_SUBTASK scratch buffer, as the reference radixSort's
// subtasks do before their redistribution callback.  One thread: the chunks
// are small and the order must be stable.
__global__ void rt_bucket_kernel(pmTaskInfo ti, pmDeviceInfo* di, pmSubtaskInfo si, pmStatus* st) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int buckets = *static_cast<const int*>(ti.taskConf);
    const int* in = static_cast<const int*>(si.memInfo[0].ptr);
    int* out = static_cast<int*>(si.memInfo[1].ptr);
    int* bins = static_cast<int*>(si.gpuContext.scratchBuffer);
    const int n = static_cast<int>(si.memInfo[0].length / 4);
    for (int b = 0; b < buckets; ++b) bins[b] = 0;
    for (int i = 0; i < n; ++i) bins[in[i] % buckets]++;
    int pos = 0;
    for (int b = 0; b < buckets; ++b)
        for (int i = 0; i < n; ++i)
            if (in[i] % buckets == b) out[pos++] = in[i];
}

extern "C" void* rt_bucket_kernel_ptr() { return reinterpret_cast<void*>(&rt_bucket_kernel); }
