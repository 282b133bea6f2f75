// prefixSum subtask kernel: inclusive scan, uint32 in -> uint64 out.
//
// Semantics: out[i] = in[0] + ... + in[i] (testSuite/prefixSum/source/code/src/
// prefixSum.cpp:47-53 serialPrefixSum, widened to 64-bit sums; the reference's
// two-task flow -- per-subtask serial scans :86-104, host scan of subtask
// totals and elemAdd :106-133 -- produces the same global inclusive scan).
//
// Design: reduce-then-scan over chunks sized for the 126 MB L2.  The input is
// cut into chunks of 2^24 elements (64 MB) and each chunk into segments of
// 16384 elements.  Launch j (j = -1 .. chunks-1, all on one stream) runs two
// kinds of 256-thread blocks side by side:
//   reduce blocks sum two segments of chunk j+1 each, reading the input from
//     HBM under an L2 evict-last policy so that it stays resident, and write
//     one uint64 per segment;
//   scan blocks scan one segment of chunk j each, from carry[j] (the sum of
//     all earlier chunks) plus the sums of the segments before theirs; they
//     read the input a second time -- mostly an L2 hit -- and stream the
//     uint64 output out under an evict-first policy.  Scan block 0 also forms
//     carry[j+1].
// Launches after the first use programmatic dependent launch: their reduce
// blocks start on SMs the previous launch has left, and their scan blocks
// wait (griddepcontrol.wait) for the previous grid's results.  No block spins
// on another block.  Each block stages its tiles through a 3-deep ring of
// 16 KB shared-memory buffers filled by single bulk async copies (one thread
// issues, an mbarrier completes), so ~48 KB per block is in flight while the
// current tile is processed.  A tile (4096 elements) is scanned with
// thread-local sums, warp shuffles and one warp scan of the 32 partial
// totals.  Measured at 2^28 elements: 13.3 bytes of HBM traffic per element
// (4 read, 8 written, ~1.3 of re-reads that missed L2).
#include <mutex>

#include "lookback.cuh"
#include "pmb_common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;                          // 16-byte loads per thread per tile
constexpr int kTile = kThreads * 4 * kRows;       // 4096 elements
constexpr int kSeg = 4 * kTile;                   // 16384 elements per scan block
constexpr size_t kChunk = size_t(1) << 24;        // 64 MB of input per launch
constexpr int kSegsPerChunk = static_cast<int>(kChunk / kSeg);  // 1024
constexpr int kReduceSegs = 2;                    // segments per reduce block
constexpr int kStages = 3;                        // tiles staged in shared memory per block
constexpr int kSmemBytes = kStages * kTile * 4;   // 48 KB (dynamic)
constexpr size_t kHeaderBytes = 256;              // {unused, error word, padding}

__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
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

// Tile staging: one thread copies the 16-byte-aligned body of tile [t0, t0 +
// kTile) clipped to `end` into shared memory with a single bulk async copy
// completing on `bar`; the reading threads take the remaining 0-3 elements of
// a ragged last tile straight from global memory.
__device__ __forceinline__ size_t tile_body(size_t t0, size_t end) {
    const size_t len = t0 + kTile <= end ? kTile : end - t0;
    return len & ~size_t(3);
}
__device__ __forceinline__ void fetch_tile(uint32_t* dst, const uint32_t* __restrict__ in, size_t t0, size_t end,
                                           uint64_t* bar, uint64_t pol) {
    const uint32_t bytes = static_cast<uint32_t>(tile_body(t0, end) * 4);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    if (bytes)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
                smem_u32(dst)),
            "l"(in + t0), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
            : "memory");
}
// Element r*1024 + 4*tid + k of a staged tile, as q[r] component k; zero past `end`.
__device__ __forceinline__ void read_tile(const uint32_t* tile, const uint32_t* __restrict__ in, size_t t0,
                                          size_t end, int tid, uint4 (&q)[kRows]) {
    if (t0 + kTile <= end) {
#pragma unroll
        for (int r = 0; r < kRows; ++r) q[r] = reinterpret_cast<const uint4*>(tile)[r * kThreads + tid];
    } else {
        const size_t body = t0 + tile_body(t0, end);
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            uint32_t e[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int off = r * (kThreads * 4) + 4 * tid + k;
                const size_t idx = t0 + off;
                e[k] = idx < body ? tile[off] : (idx < end ? in[idx] : 0u);
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

__global__ void __launch_bounds__(kThreads)
scan_chunks_kernel(const uint32_t* __restrict__ in, uint64_t* __restrict__ out, size_t n, int j, int scan_blocks,
                   uint64_t* __restrict__ carry, uint64_t* __restrict__ sums, uint32_t* __restrict__ hdr) {
    extern __shared__ __align__(128) unsigned char smem[];  // kStages staged tiles
    __shared__ uint64_t s_bar[kStages];
    __shared__ uint64_t s_red[2][kThreads / 32];
    __shared__ uint64_t s_wt[2][kRows][kThreads / 32];
    __shared__ uint64_t s_tot[2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t* tiles = reinterpret_cast<uint32_t*>(smem);
    const bool reducer = static_cast<int>(blockIdx.x) >= scan_blocks;
    // The next launch may start filling SMs as this one drains (programmatic
    // dependent launch); its scan blocks wait for this grid before reading.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    if (tid == 0) {
        if (reducer && j < 0 && blockIdx.x == static_cast<unsigned>(scan_blocks)) {
            carry[0] = 0;
            hdr[1] = 0;  // error word (set below only if a staging wait expires)
        }
        for (int st = 0; st < kStages; ++st) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar[st])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    // The block's range [r0, r1) is staged tile by tile through the ring.
    size_t r0, r1;
    if (reducer) {
        const size_t c1 = static_cast<size_t>(j + 1) * kChunk;
        const size_t c1_end = c1 + kChunk < n ? c1 + kChunk : n;
        r0 = c1 + static_cast<size_t>(blockIdx.x - scan_blocks) * kReduceSegs * kSeg;
        r1 = r0 + static_cast<size_t>(kReduceSegs) * kSeg < c1_end ? r0 + static_cast<size_t>(kReduceSegs) * kSeg
                                                                     : c1_end;
    } else {
        r0 = static_cast<size_t>(j) * kChunk + static_cast<size_t>(blockIdx.x) * kSeg;
        r1 = r0 + kSeg < n ? r0 + kSeg : n;
    }
    const int ntiles = static_cast<int>((r1 - r0 + kTile - 1) / kTile);
    const uint64_t pin = reducer ? policy_evict_last() : policy_evict_first();
    if (tid == 0)
        for (int t = 0; t < kStages && t < ntiles; ++t)
            fetch_tile(tiles + t * kTile, in, r0 + static_cast<size_t>(t) * kTile, r1, &s_bar[t], pin);
    bool ok = true;

    if (reducer) {
        // ---- reduce: one sum per kSeg segment of chunk j+1 ----
        uint64_t acc = 0;
        for (int t = 0; t < ntiles; ++t) {
            const int st = t % kStages;
            const size_t t0 = r0 + static_cast<size_t>(t) * kTile;
            ok &= mbar_wait(smem_u32(&s_bar[st]), (t / kStages) & 1);
            uint4 q[kRows];
            read_tile(tiles + st * kTile, in, t0, r1, tid, q);
#pragma unroll
            for (int r = 0; r < kRows; ++r) acc += static_cast<uint64_t>(q[r].x) + q[r].y + q[r].z + q[r].w;
            __syncthreads();  // every thread has read stage st
            if (tid == 0 && t + kStages < ntiles)
                fetch_tile(tiles + st * kTile, in, t0 + static_cast<size_t>(kStages) * kTile, r1, &s_bar[st], pin);
            if ((t + 1) % (kSeg / kTile) == 0 || t + 1 == ntiles) {
                const uint64_t total = block_sum(acc, s_red[(t / (kSeg / kTile)) & 1]);
                const size_t seg = (t0 - static_cast<size_t>(j + 1) * kChunk) / kSeg;
                if (tid == 0) sums[static_cast<size_t>(j + 1) * kSegsPerChunk + seg] = total;
                acc = 0;
            }
        }
    } else {
        // ---- scan one segment of chunk j ----
        // The previous launch wrote this chunk's segment sums and carry[j].
        asm volatile("griddepcontrol.wait;" ::: "memory");
        const int seg = blockIdx.x;
        const size_t c0 = static_cast<size_t>(j) * kChunk;
        const uint64_t* cs = sums + static_cast<size_t>(j) * kSegsPerChunk;
        const int nsegs = static_cast<int>(((c0 + kChunk < n ? c0 + kChunk : n) - c0 + kSeg - 1) / kSeg);
        uint64_t before = 0, all = 0;
        for (int t = tid; t < nsegs; t += kThreads) {
            const uint64_t x = cs[t];
            all += x;
            if (t < seg) before += x;
        }
        const uint64_t cj = carry[j];
        uint64_t base = cj + block_sum(before, s_red[0]);
        if (seg == 0) {
            const uint64_t tot = block_sum(all, s_red[1]);
            if (tid == 0) carry[j + 1] = cj + tot;
        }
        const uint64_t pout = policy_evict_first();
        for (int t = 0; t < ntiles; ++t) {
            const int st = t % kStages, par = t & 1;
            const size_t t0 = r0 + static_cast<size_t>(t) * kTile;
            ok &= mbar_wait(smem_u32(&s_bar[st]), (t / kStages) & 1);
            uint4 cur[kRows];
            read_tile(tiles + st * kTile, in, t0, r1, tid, cur);
            uint64_t lane_excl[kRows];  // this thread's offset inside its warp's row piece
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const uint64_t own = static_cast<uint64_t>(cur[r].x) + cur[r].y + cur[r].z + cur[r].w;
                const uint64_t incl = pmb::warp_inclusive_scan_u64(own, lane);
                lane_excl[r] = incl - own;
                if (lane == 31) s_wt[par][r][warp] = incl;
            }
            __syncthreads();  // s_wt complete; every thread has read stage st
            if (tid == 0 && t + kStages < ntiles)
                fetch_tile(tiles + st * kTile, in, t0 + static_cast<size_t>(kStages) * kTile, r1, &s_bar[st], pin);
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
                    st_u64x2(out + idx, o0, o1, pout);
                    st_u64x2(out + idx + 2, o2, o3, pout);
                } else {
                    const uint64_t o[4] = {o0, o1, o2, o3};
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (idx + k < r1) out[idx + k] = o[k];
                }
            }
            base += s_tot[par];
        }
    }
    if (!ok) atomicOr(&hdr[1], pmb::kErrLookbackTimeout);
}

constexpr size_t num_chunks(size_t n) { return (n + kChunk - 1) / kChunk; }
constexpr int segs_of_chunk(size_t n, size_t c) {
    return static_cast<int>(((c + 1) * kChunk < n ? kChunk : n - c * kChunk) + kSeg - 1) / kSeg;
}

}  // namespace

namespace pmb {

constexpr size_t scan_scratch_need(size_t n) {
    return kHeaderBytes + 8 * (num_chunks(n) + 1) + 8 * num_chunks(n) * kSegsPerChunk;
}

size_t scan_scratch_bytes(size_t n) { return scan_scratch_need(n); }

// Shared by the public entry points: validates and runs the launch sequence.
// The kernels write every scratch word they read, so nothing is cleared first.
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
        attr_err = cudaFuncSetAttribute(scan_chunks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    });
    PMB_CUDA_TRY(attr_err);
    uint32_t* hdr = static_cast<uint32_t*>(d_scratch);
    const size_t nc = num_chunks(n);
    uint64_t* carry = reinterpret_cast<uint64_t*>(static_cast<char*>(d_scratch) + kHeaderBytes);
    uint64_t* sums = carry + (nc + 1);
    for (long long j = -1; j < static_cast<long long>(nc); ++j) {
        const int sb = j >= 0 ? segs_of_chunk(n, static_cast<size_t>(j)) : 0;
        const int rb = j + 1 < static_cast<long long>(nc)
                           ? (segs_of_chunk(n, static_cast<size_t>(j + 1)) + kReduceSegs - 1) / kReduceSegs
                           : 0;
        // Launch -1 waits for all earlier work on the stream (the input may come
        // from it); later launches overlap their predecessor's tail.
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(sb + rb);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = kSmemBytes;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = j >= 0 ? 1 : 0;
        PMB_CUDA_TRY(
            cudaLaunchKernelEx(&cfg, scan_chunks_kernel, d_in, d_out, n, static_cast<int>(j), sb, carry, sums, hdr));
    }
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
    // The shared array keeps the previous call's contents; the kernels write
    // every word of it that they read (the carries and segment sums) first.
    return pmb::scan_launch(d_in, d_out, n, scratch, kNoAllocScratchBytes, static_cast<cudaStream_t>(stream));
}
