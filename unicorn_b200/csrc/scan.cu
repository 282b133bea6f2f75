// prefixSum subtask kernel: single-pass inclusive scan, uint32 in -> uint64 out.
//
// Semantics: out[i] = in[0] + ... + in[i] (testSuite/prefixSum/source/code/src/
// prefixSum.cpp:47-53 serialPrefixSum, widened to 64-bit sums; the reference's
// two-task flow -- per-subtask serial scans :86-104, host scan of subtask
// totals and elemAdd :106-133 -- produces the same global inclusive scan).
//
// Design (decoupled look-back, one launch): each 256-thread CTA takes the next
// 4096-element tile from a global counter (so every tile it waits on belongs
// to a CTA that is already running), scans it in registers (4 coalesced
// 16-byte loads per thread, thread-local scans, warp shuffles, one 32-value
// warp scan of warp totals), publishes its tile aggregate, and warp 0 walks
// back over predecessors 32 tiles at a time until it meets an inclusive
// prefix.  Status words pack {flag:2, value:62}, so a relaxed 64-bit load sees
// flag and value together.  Every input byte is read once and every output
// byte written once: 12 bytes of HBM traffic per element.
#include <mutex>

#include "lookback.cuh"
#include "pmb_common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;                     // 16-byte loads per thread
constexpr int kTile = kThreads * 4 * kRows;  // 4096 elements
constexpr uint64_t kValMask = (1ull << 62) - 1;
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr size_t kHeaderBytes = 256;  // {tile counter, error word, padding}

__global__ void __launch_bounds__(kThreads)
scan_u32_u64_kernel(const uint32_t* __restrict__ in, uint64_t* __restrict__ out, size_t n,
                    uint32_t* __restrict__ hdr, uint64_t* __restrict__ status) {
    __shared__ uint64_t s_wt[kRows][kThreads / 32];
    __shared__ uint64_t s_excl;
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(&hdr[0], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = static_cast<size_t>(tile) * kTile;

    uint64_t v[kRows][4];
    uint64_t lane_incl[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const size_t idx = base + static_cast<size_t>(r) * (kThreads * 4) + 4 * tid;
        if (idx + 3 < n) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(in + idx));
            v[r][0] = q.x; v[r][1] = q.y; v[r][2] = q.z; v[r][3] = q.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) v[r][j] = idx + j < n ? in[idx + j] : 0u;
        }
        v[r][1] += v[r][0];
        v[r][2] += v[r][1];
        v[r][3] += v[r][2];
        lane_incl[r] = pmb::warp_inclusive_scan_u64(v[r][3], lane);
        if (lane == 31) s_wt[r][warp] = lane_incl[r];
    }
    __syncthreads();

    if (warp == 0) {
        // kRows * 8 warps == 32 partial totals, in element order (row-major).
        const uint64_t x = s_wt[lane >> 3][lane & 7];
        const uint64_t inc = pmb::warp_inclusive_scan_u64(x, lane);
        s_wt[lane >> 3][lane & 7] = inc - x;
        const uint64_t agg = __shfl_sync(0xffffffffu, inc, 31);
        uint64_t excl = 0;
        if (tile == 0) {
            if (lane == 0) pmb::st_relaxed_u64(&status[0], kFlagInc | (agg & kValMask));
        } else {
            if (lane == 0) pmb::st_relaxed_u64(&status[tile], kFlagAgg | (agg & kValMask));
            long long cur = static_cast<long long>(tile) - 1;
            bool gave_up = false;
            for (;;) {
                const long long idx = cur - lane;
                uint64_t s = idx >= 0 ? pmb::ld_relaxed_u64(&status[idx]) : kFlagInc;
                if (!gave_up) {
                    uint32_t polls = 0;
                    while (__any_sync(0xffffffffu, (s >> 62) == 0)) {
                        if (++polls > pmb::kSpinLimit) {
                            gave_up = true;
                            break;
                        }
                        __nanosleep(100);
                        if ((s >> 62) == 0) s = pmb::ld_relaxed_u64(&status[idx]);
                    }
                }
                const uint32_t incmask = __ballot_sync(0xffffffffu, (s >> 62) == 2);
                uint64_t val = s & kValMask;
                if (incmask) {
                    if (lane > __ffs(incmask) - 1) val = 0;
                    excl += pmb::warp_sum_u64(val);
                    break;
                }
                excl += pmb::warp_sum_u64(val);
                cur -= 32;
            }
            if (lane == 0) {
                if (gave_up) atomicOr(&hdr[1], pmb::kErrLookbackTimeout);
                pmb::st_relaxed_u64(&status[tile], kFlagInc | ((excl + agg) & kValMask));
            }
        }
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();

    const uint64_t texcl = s_excl;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const uint64_t add = texcl + s_wt[r][warp] + lane_incl[r] - v[r][3];
        const size_t idx = base + static_cast<size_t>(r) * (kThreads * 4) + 4 * tid;
        if (idx + 3 < n) {
            ulonglong2* o = reinterpret_cast<ulonglong2*>(out + idx);
            o[0] = make_ulonglong2(v[r][0] + add, v[r][1] + add);
            o[1] = make_ulonglong2(v[r][2] + add, v[r][3] + add);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (idx + j < n) out[idx + j] = v[r][j] + add;
        }
    }
}

size_t num_tiles(size_t n) { return (n + kTile - 1) / kTile; }

}  // namespace

namespace pmb {

size_t scan_scratch_bytes(size_t n) { return kHeaderBytes + 8 * num_tiles(n); }

// Shared by the public entry points: validates, clears the scratch and launches.
int scan_launch(const uint32_t* d_in, uint64_t* d_out, size_t n, void* d_scratch, size_t scratch_bytes,
                cudaStream_t s, bool clear_with_memset) {
    if (n == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(d_in && d_out && d_scratch, "null pointer");
    PMB_CHECK_ARG(n <= (1ull << 30), "scan length %zu above 2^30 (62-bit status sums)", n);
    PMB_CHECK_ARG(((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15) == 0,
                  "scan input/output must be 16-byte aligned");
    PMB_CHECK_ARG((reinterpret_cast<uintptr_t>(d_scratch) & 15) == 0, "scratch must be 16-byte aligned");
    const size_t need = scan_scratch_bytes(n);
    if (scratch_bytes < need)
        return fail(PMB_BEYOND_LIMITS, "scan scratch %zu bytes, need %zu", scratch_bytes, need);
    if (clear_with_memset) PMB_CUDA_TRY(cudaMemsetAsync(d_scratch, 0, need, s));
    uint32_t* hdr = static_cast<uint32_t*>(d_scratch);
    uint64_t* status = reinterpret_cast<uint64_t*>(static_cast<char*>(d_scratch) + kHeaderBytes);
    scan_u32_u64_kernel<<<static_cast<unsigned>(num_tiles(n)), kThreads, 0, s>>>(d_in, d_out, n, hdr, status);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

}  // namespace pmb

extern "C" size_t pmb_scan_scratch_bytes(size_t n) { return pmb::scan_scratch_bytes(n); }

extern "C" int pmb_inclusive_scan_u32_u64(const uint32_t* d_in, uint64_t* d_out, size_t n, void* d_scratch,
                                          size_t scratch_bytes, void* stream) {
    return pmb::scan_launch(d_in, d_out, n, d_scratch, scratch_bytes, static_cast<cudaStream_t>(stream), true);
}

extern "C" int pmb_scratch_error(const void* d_scratch, uint32_t* error_out) {
    PMB_CHECK_ARG(d_scratch && error_out, "null pointer");
    PMB_CUDA_TRY(cudaMemcpy(error_out, static_cast<const uint32_t*>(d_scratch) + 1, sizeof(uint32_t),
                            cudaMemcpyDeviceToHost));
    return PMB_SUCCESS;
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers may not allocate device memory at
// all: a pm:: subtask_gpu_custom callback must only enqueue work on the stream
// it is given (cudaMalloc and cudaFree synchronise the device and would stall
// the stub's pipeline of in-flight subtasks), and services that fix their
// memory budget up front cannot let a library grow it behind their back.  For
// them the scan's look-back scratch lives in a fixed device array that every
// GPU loading this library holds until the process exits.
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(1) << 20;  // 1 MiB per device
__device__ __align__(256) unsigned char g_noalloc_scan_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_scan_scratch on the current device, looked up
// once per device (the host-side name of the array is not a device address).
int noalloc_scratch(void** out) {
    int dev = 0;
    PMB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return pmb::fail(PMB_BEYOND_LIMITS, "device %d beyond %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        PMB_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scan_scratch));
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return PMB_SUCCESS;
}

}  // namespace

static_assert(PMB_SCAN_NOALLOC_MAX_ELEMS == (kNoAllocScratchBytes - kHeaderBytes) / 8 * kTile,
              "header limit must match the scratch array");

extern "C" int pmb_inclusive_scan_u32_u64_noalloc(const uint32_t* d_in, uint64_t* d_out, size_t n, void* stream) {
    if (n == 0) return PMB_SUCCESS;
    if (n > PMB_SCAN_NOALLOC_MAX_ELEMS)
        return pmb::fail(PMB_BEYOND_LIMITS,
                         "pmb_inclusive_scan_u32_u64_noalloc: %zu elements exceed the fixed scratch limit of %llu; "
                         "use pmb_inclusive_scan_u32_u64 with caller-provided scratch",
                         n, static_cast<unsigned long long>(PMB_SCAN_NOALLOC_MAX_ELEMS));
    void* scratch = nullptr;
    const int st = noalloc_scratch(&scratch);
    if (st != PMB_SUCCESS) return st;
    // The shared array keeps the previous call's contents: scan_launch clears
    // the header and the status words this call uses before the kernel runs.
    return pmb::scan_launch(d_in, d_out, n, scratch, kNoAllocScratchBytes, static_cast<cudaStream_t>(stream), true);
}
