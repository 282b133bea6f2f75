// prefixSum subtask kernel: inclusive scan, uint32 in -> uint64 out.
//
// Semantics: out[i] = in[0] + ... + in[i] (testSuite/prefixSum/source/code/src/
// prefixSum.cpp:47-53 serialPrefixSum, widened to 64-bit sums; the reference's
// two-task flow -- per-subtask serial scans :86-104, host scan of subtask
// totals and elemAdd :106-133 -- produces the same global inclusive scan).
//
// Design: one launch, single pass, decoupled look-back (Merrill and Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back", 2016).  Each
// 256-thread block takes the next 16384-element tile from a global counter
// (so every tile it waits on belongs to a block that started earlier), stages
// the tile in shared memory with four 16 KB bulk async copies (one mbarrier
// each), sums it, and publishes the sum in the tile's 64-bit status word
// (2-bit flag | 62-bit value: AGGREGATE, or INCLUSIVE for tile 0).  Warp 0
// then reads the status words of the 32 preceding tiles at once, adds the
// aggregates back to the nearest inclusive prefix (waiting -- boundedly -- only
// for tiles in between that have not published yet), and publishes the tile's
// own inclusive prefix.  The block then scans the staged tile from that
// offset: per 4096-element sub-tile, thread-local sums of four elements, warp
// shuffle scans of the 32 row pieces and one warp scan of their totals, and
// coalesced 16-byte stores of the uint64 results.  HBM traffic: 4 bytes read
// and 8 written per element, plus 8 bytes of status per 16384 elements.  The
// 62-bit status values hold any sum of n <= 2^30 uint32 values (< 2^62).
#include <algorithm>
#include <mutex>

#include "lookback.cuh"
#include "pmb_common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;                          // 16-byte reads per thread per sub-tile
constexpr int kSub = kThreads * 4 * kRows;        // 4096 elements per staged sub-tile
constexpr int kSubs = 4;                          // sub-tiles per block tile
constexpr int kTile = kSub * kSubs;               // 16384 elements per block
constexpr int kSmemBytes = kTile * 4;             // 64 KB (dynamic)
constexpr size_t kHeaderBytes = 256;              // {tile counter, error word, padding}
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValueMask = (1ull << 62) - 1;

__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void st_u64x2(uint64_t* p, uint64_t a, uint64_t b, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.u64 [%0], {%1, %2}, %3;" ::"l"(p), "l"(a), "l"(b), "l"(pol) : "memory");
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bounded wait for an mbarrier phase; false once the poll limit is reached.
constexpr uint32_t kWaitPolls = 1u << 21;  // each poll suspends for at most ~1 us
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitPolls; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Sub-tile staging: one thread copies the 16-byte-aligned body of sub-tile
// [t0, t0 + kSub) clipped to `end` into shared memory with a single bulk async
// copy completing on `bar`; the reading threads take the remaining 0-3
// elements of a ragged last sub-tile straight from global memory.
__device__ __forceinline__ size_t sub_body(size_t t0, size_t end) {
    const size_t len = t0 + kSub <= end ? kSub : end - t0;
    return len & ~size_t(3);
}
__device__ __forceinline__ void fetch_sub(uint32_t* dst, const uint32_t* __restrict__ in, size_t t0, size_t end,
                                          uint64_t* bar, uint64_t pol) {
    const uint32_t bytes = static_cast<uint32_t>(sub_body(t0, end) * 4);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    if (bytes)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
                smem_u32(dst)),
            "l"(in + t0), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
            : "memory");
}
// Element r*1024 + 4*tid + k of a staged sub-tile, as q[r] component k; zero past `end`.
__device__ __forceinline__ void read_sub(const uint32_t* sub, const uint32_t* __restrict__ in, size_t t0,
                                         size_t end, int tid, uint4 (&q)[kRows]) {
    if (t0 + kSub <= end) {
#pragma unroll
        for (int r = 0; r < kRows; ++r) q[r] = reinterpret_cast<const uint4*>(sub)[r * kThreads + tid];
    } else {
        const size_t body = t0 + sub_body(t0, end);
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            uint32_t e[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int off = r * (kThreads * 4) + 4 * tid + k;
                const size_t idx = t0 + off;
                e[k] = idx < body ? sub[off] : (idx < end ? in[idx] : 0u);
            }
            q[r] = make_uint4(e[0], e[1], e[2], e[3]);
        }
    }
}

__device__ __forceinline__ uint64_t block_sum(uint64_t v, uint64_t* s_red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = pmb::warp_sum_u64(v);
    __syncthreads();  // s_red may still be read from an earlier use
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    uint64_t t = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) t += s_red[w];
    return t;
}

// Exclusive prefix of tile `tile` from the status words of its predecessors,
// run by one full warp.  Lane i looks at tile (base - i); a round sums the
// aggregates of the tiles up to the nearest published inclusive prefix, and
// waits only while one of those tiles has published nothing yet.  Sets
// *gave_up (and counts the unpublished tiles as 0) once the poll limit is hit.
__device__ __forceinline__ uint64_t lookback(const uint64_t* status, long long tile, int lane, bool* gave_up) {
    uint64_t excl = 0;
    for (long long base = tile - 1;; base -= 32) {
        const long long idx = base - lane;
        uint64_t s = idx >= 0 ? pmb::ld_relaxed_u64(&status[idx]) : kFlagInc;
        uint32_t inc_mask, upto;
        for (uint32_t polls = 0;; ++polls) {
            inc_mask = __ballot_sync(0xffffffffu, (s >> 62) == 2);
            // Lanes up to and including the first inclusive prefix (all 32 if none).
            upto = inc_mask ? (inc_mask ^ (inc_mask - 1)) : 0xffffffffu;
            const uint32_t pending = __ballot_sync(0xffffffffu, (s >> 62) == 0) & upto;
            if (!pending) break;
            if (polls >= pmb::kSpinLimit) {
                *gave_up = true;
                break;
            }
            __nanosleep(32);
            if ((pending >> lane) & 1u) s = pmb::ld_relaxed_u64(&status[idx]);
        }
        excl += pmb::warp_sum_u64(((upto >> lane) & 1u) ? (s & kValueMask) : 0);
        if (inc_mask || *gave_up) return excl;
    }
}

__global__ void __launch_bounds__(kThreads, 3)
scan_lookback_kernel(const uint32_t* __restrict__ in, uint64_t* __restrict__ out, size_t n,
                     uint64_t* __restrict__ status, uint32_t* __restrict__ hdr) {
    extern __shared__ __align__(128) unsigned char smem[];  // the block's staged tile
    __shared__ uint64_t s_bar[kSubs];
    __shared__ uint64_t s_red[kThreads / 32];
    __shared__ uint64_t s_wt[2][kRows][kThreads / 32];
    __shared__ uint64_t s_tot[2];
    __shared__ uint64_t s_excl;
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t* stage = reinterpret_cast<uint32_t*>(smem);
    const uint64_t pol = policy_evict_first();  // input and output stream through L2 once

    if (tid == 0) {
        s_tile = atomicAdd(&hdr[0], 1u);
        for (int st = 0; st < kSubs; ++st) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar[st])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const size_t tile = s_tile;
    const size_t r0 = tile * kTile;
    const size_t r1 = r0 + kTile < n ? r0 + kTile : n;
    const int nsub = static_cast<int>((r1 - r0 + kSub - 1) / kSub);
    if (tid == 0)
        for (int st = 0; st < nsub; ++st)
            fetch_sub(stage + st * kSub, in, r0 + static_cast<size_t>(st) * kSub, r1, &s_bar[st], pol);

    // ---- the tile's sum, published as soon as it is known ----
    bool ok = true;
    uint64_t acc = 0;
    for (int st = 0; st < nsub; ++st) {
        ok &= mbar_wait(smem_u32(&s_bar[st]), 0);
        uint4 q[kRows];
        read_sub(stage + st * kSub, in, r0 + static_cast<size_t>(st) * kSub, r1, tid, q);
#pragma unroll
        for (int r = 0; r < kRows; ++r) acc += static_cast<uint64_t>(q[r].x) + q[r].y + q[r].z + q[r].w;
    }
    const uint64_t agg = block_sum(acc, s_red);
    if (warp == 0) {
        uint64_t excl = 0;
        if (tile == 0) {
            if (lane == 0) pmb::st_relaxed_u64(&status[0], kFlagInc | agg);
        } else {
            if (lane == 0) pmb::st_relaxed_u64(&status[tile], kFlagAgg | agg);
            bool gave_up = false;
            excl = lookback(status, static_cast<long long>(tile), lane, &gave_up);
            if (lane == 0) {
                pmb::st_relaxed_u64(&status[tile], kFlagInc | ((excl + agg) & kValueMask));
                if (gave_up) atomicOr(&hdr[1], pmb::kErrLookbackTimeout);
            }
        }
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();

    // ---- scan the staged tile from its exclusive prefix ----
    uint64_t base = s_excl;
    for (int st = 0; st < nsub; ++st) {
        const int par = st & 1;
        const size_t t0 = r0 + static_cast<size_t>(st) * kSub;
        uint4 cur[kRows];
        read_sub(stage + st * kSub, in, t0, r1, tid, cur);
        uint64_t lane_excl[kRows];  // this thread's offset inside its warp's row piece
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            const uint64_t own = static_cast<uint64_t>(cur[r].x) + cur[r].y + cur[r].z + cur[r].w;
            const uint64_t incl = pmb::warp_inclusive_scan_u64(own, lane);
            lane_excl[r] = incl - own;
            if (lane == 31) s_wt[par][r][warp] = incl;
        }
        __syncthreads();  // s_wt[par] complete
        if (warp == 0) {
            // kRows * 8 warps == 32 partial totals, in element order (row-major).
            const uint64_t x = s_wt[par][lane >> 3][lane & 7];
            const uint64_t inc = pmb::warp_inclusive_scan_u64(x, lane);
            s_wt[par][lane >> 3][lane & 7] = inc - x;
            if (lane == 31) s_tot[par] = inc;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            const uint64_t o0 = base + s_wt[par][r][warp] + lane_excl[r] + cur[r].x;
            const uint64_t o1 = o0 + cur[r].y, o2 = o1 + cur[r].z, o3 = o2 + cur[r].w;
            const size_t idx = t0 + static_cast<size_t>(r) * (kThreads * 4) + 4 * tid;
            if (idx + 3 < r1) {
                st_u64x2(out + idx, o0, o1, pol);
                st_u64x2(out + idx + 2, o2, o3, pol);
            } else {
                const uint64_t o[4] = {o0, o1, o2, o3};
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (idx + k < r1) out[idx + k] = o[k];
            }
        }
        // s_wt[par] and s_tot[par] are rewritten two sub-tiles later, after the
        // first barrier of the next sub-tile has ordered these reads.
        base += s_tot[par];
    }
    if (!ok) atomicOr(&hdr[1], pmb::kErrLookbackTimeout);
}

constexpr size_t num_tiles(size_t n) { return (n + kTile - 1) / kTile; }

}  // namespace

namespace pmb {

constexpr size_t scan_scratch_need(size_t n) { return kHeaderBytes + 8 * num_tiles(n); }

size_t scan_scratch_bytes(size_t n) { return scan_scratch_need(n); }

// Shared by the public entry points: validates, clears the tile counter, the
// error word and the status words, and launches the single pass.
int scan_launch(const uint32_t* d_in, uint64_t* d_out, size_t n, void* d_scratch, size_t scratch_bytes,
                cudaStream_t s) {
    if (n == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(d_in && d_out && d_scratch, "null pointer");
    PMB_CHECK_ARG(n <= (1ull << 30), "scan length %zu above 2^30", n);
    PMB_CHECK_ARG(((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15) == 0,
                  "scan input/output must be 16-byte aligned");
    PMB_CHECK_ARG((reinterpret_cast<uintptr_t>(d_scratch) & 15) == 0, "scratch must be 16-byte aligned");
    const size_t need = scan_scratch_bytes(n);
    if (scratch_bytes < need)
        return fail(PMB_BEYOND_LIMITS, "scan scratch %zu bytes, need %zu", scratch_bytes, need);
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(scan_lookback_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    });
    PMB_CUDA_TRY(attr_err);
    PMB_CUDA_TRY(cudaMemsetAsync(d_scratch, 0, need, s));
    uint32_t* hdr = static_cast<uint32_t*>(d_scratch);
    uint64_t* status = reinterpret_cast<uint64_t*>(static_cast<char*>(d_scratch) + kHeaderBytes);
    const size_t tiles = num_tiles(n);
    scan_lookback_kernel<<<static_cast<unsigned>(tiles), kThreads, kSmemBytes, s>>>(d_in, d_out, n, status, hdr);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

}  // namespace pmb

extern "C" size_t pmb_scan_scratch_bytes(size_t n) { return pmb::scan_scratch_bytes(n); }

extern "C" int pmb_inclusive_scan_u32_u64(const uint32_t* d_in, uint64_t* d_out, size_t n, void* d_scratch,
                                          size_t scratch_bytes, void* stream) {
    return pmb::scan_launch(d_in, d_out, n, d_scratch, scratch_bytes, static_cast<cudaStream_t>(stream));
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
// them the scan's scratch (tile counter, error word, tile status words) lives
// in a fixed device array that every GPU loading this library holds until the
// process exits.
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

static_assert(pmb::scan_scratch_need(PMB_SCAN_NOALLOC_MAX_ELEMS) <= kNoAllocScratchBytes,
              "the header's element limit must fit the scratch array");

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
    // The shared array keeps the previous call's contents; scan_launch clears
    // the counter, the error word and the status words on the stream first.
    return pmb::scan_launch(d_in, d_out, n, scratch, kNoAllocScratchBytes, static_cast<cudaStream_t>(stream));
}

extern "C" int pmb_scan_noalloc_error(uint32_t* error_out) {
    PMB_CHECK_ARG(error_out, "null pointer");
    void* scratch = nullptr;
    const int st = noalloc_scratch(&scratch);
    if (st != PMB_SUCCESS) return st;
    PMB_CUDA_TRY(cudaMemcpy(error_out, static_cast<const uint32_t*>(scratch) + 1, sizeof(uint32_t),
                            cudaMemcpyDeviceToHost));
    return PMB_SUCCESS;
}

// ---------------------------------------------------------------------------
// The prefix sum's second task: add the total of the preceding slices to
// every element of a slice (elemAdd_cuda, testSuite/prefixSum/source/code/
// src/prefixSumCUDA.cu:143-158, widened to uint64).  The total is read on the
// device, so the task's data dependencies stay on the stream.
namespace {

__global__ void __launch_bounds__(256)
add_scalar_kernel(uint64_t* __restrict__ d, size_t n, const uint64_t* __restrict__ scalar) {
    const uint64_t v = *scalar;
    const size_t n2 = n / 2;
    ulonglong2* d2 = reinterpret_cast<ulonglong2*>(d);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n2;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        ulonglong2 x = d2[i];
        x.x += v;
        x.y += v;
        d2[i] = x;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) d[n - 1] += v;
}

}  // namespace

extern "C" int pmb_add_u64_scalar(uint64_t* d_data, size_t n, const uint64_t* d_scalar, void* stream) {
    if (n == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(d_data && d_scalar, "null pointer");
    PMB_CHECK_ARG((reinterpret_cast<uintptr_t>(d_data) & 15) == 0, "data must be 16-byte aligned");
    int dev = 0, sms = 148;
    PMB_CUDA_TRY(cudaGetDevice(&dev));
    PMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t want = (n / 2 + 255) / 256;
    const unsigned grid = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(want, static_cast<size_t>(sms) * 8)));
    add_scalar_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_data, n, d_scalar);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}
