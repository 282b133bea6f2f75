// Sentinel compression of reduction outputs for their trip to the host.
//
// The reference compresses a GPU subtask's reduction output before copying
// it back when most of it is the sentinel value zero
// (source/code/src/pmCudaInterface.cu:380-472 CompressForSentinel: a thrust
// count and two copy_ifs; pmExecutionStub.cpp:3850-3950 decides and
// uncompresses; thresholds in pmInternalDefinitions.h:223-224).  The
// compressed form is the one its uncompress side reads
// (pmExecutionStub.cpp:3885-3908): a uint32 count, then the count non-zero
// elements, then their count uint32 indices, in index order; it is produced
// only when count < 0.4 x elements.
//
// Three launches on one stream, no host synchronisation: (1) each
// 4096-element block counts its non-zero elements; (2) one CTA scans the
// block counts into offsets, writes the count word and decides; (3) when the
// compressed form is small enough, each block writes its non-zero elements
// and indices at its offset (warp ballots keep index order).  Otherwise only
// the count word is written and the caller copies the data as it is.
// Elements are stored as 32-bit words (two per 8-byte element) because the
// 4-byte count leaves 8-byte elements 4-byte aligned.  pmb_sentinel_expand
// restores an array on the host: zero everywhere, the listed elements at
// their indices.
#include <cstring>

#include "pmb_common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kBlock = kThreads * kItems;  // elements per block
constexpr double kMaxNonSentinels = 0.4;   // CUDA_SENTINEL_COMPRESSION_MAX_NON_SENTINELS

template <typename T>
__global__ void __launch_bounds__(kThreads)
sentinel_count_kernel(const T* __restrict__ src, size_t n, uint32_t* __restrict__ counts) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t w0 = static_cast<size_t>(blockIdx.x) * kBlock + static_cast<size_t>(warp) * (kItems * 32);
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const size_t i = w0 + static_cast<size_t>(k) * 32 + lane;
        c += (i < n && src[i] != T(0)) ? 1u : 0u;
    }
    __shared__ uint32_t s[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) s[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kThreads / 32; ++w) t += s[w];
        counts[blockIdx.x] = t;
    }
}

// Exclusive scan of the block counts in place; header[0] = the total;
// *flag = 1 when the total is below the compression limit.
__global__ void __launch_bounds__(1024)
sentinel_scan_kernel(uint32_t* __restrict__ counts, uint32_t nblocks, double limit, uint32_t* __restrict__ header,
                     uint32_t* __restrict__ flag) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < nblocks; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t x = i < nblocks ? counts[i] : 0u;
        uint32_t inc = x;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        uint32_t total = 0;
        if (warp == 0) {
            const uint32_t w = s_warp[lane];
            uint32_t wi = w;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += y;
            }
            s_warp[lane] = wi - w;
            total = __shfl_sync(0xffffffffu, wi, 31);
        }
        const uint32_t carry = s_carry;
        __syncthreads();
        if (i < nblocks) counts[i] = carry + s_warp[warp] + inc - x;
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        header[0] = s_carry;
        *flag = static_cast<double>(s_carry) < limit ? 1u : 0u;
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
sentinel_compact_kernel(const T* __restrict__ src, size_t n, const uint32_t* __restrict__ offsets,
                        const uint32_t* __restrict__ flag, uint32_t* __restrict__ dst) {
    if (*flag == 0) return;
    constexpr int W = sizeof(T) / 4;  // 32-bit words per element
    const uint32_t count = dst[0];
    uint32_t* values = dst + 1;
    uint32_t* indices = dst + 1 + static_cast<size_t>(count) * W;
    __shared__ uint32_t s_warp[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Warp w owns elements [b0 + 512 w, b0 + 512 (w + 1)), 16 rounds of 32:
    // index order is warp-major, then round, then lane.
    const size_t w0 = static_cast<size_t>(blockIdx.x) * kBlock + static_cast<size_t>(warp) * (kItems * 32);
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const size_t i = w0 + static_cast<size_t>(k) * 32 + lane;
        mine += __popc(__ballot_sync(0xffffffffu, i < n && src[i] != T(0)));
    }
    if (lane == 0) s_warp[warp] = mine;
    __syncthreads();
    uint32_t pos = offsets[blockIdx.x];
    for (int w = 0; w < warp; ++w) pos += s_warp[w];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const size_t i = w0 + static_cast<size_t>(k) * 32 + lane;
        const T v = i < n ? src[i] : T(0);
        const bool nz = i < n && v != T(0);
        const uint32_t m = __ballot_sync(0xffffffffu, nz);
        if (nz) {
            const uint32_t p = pos + __popc(m & ((1u << lane) - 1u));
            uint32_t words[W];
            memcpy(words, &v, sizeof(T));
#pragma unroll
            for (int h = 0; h < W; ++h) values[static_cast<size_t>(p) * W + h] = words[h];
            indices[p] = static_cast<uint32_t>(i);
        }
        pos += __popc(m);
    }
}

size_t elem_size(int type) {
    switch (type) {
        case 0: case 1: case 4: return 4;  // INTS, UNSIGNED_INTS, FLOATS
        case 2: case 3: case 5: return 8;  // LONGS, UNSIGNED_LONGS, DOUBLES
        default: return 0;
    }
}

size_t align16(size_t b) { return (b + 15) & ~size_t(15); }
uint32_t num_blocks(size_t n) { return static_cast<uint32_t>((n + kBlock - 1) / kBlock); }

template <typename T>
int compress_t(const void* d_src, size_t n, void* d_dst, void* d_scratch, cudaStream_t s) {
    const uint32_t nb = num_blocks(n);
    uint32_t* counts = static_cast<uint32_t*>(d_scratch);
    uint32_t* flag = counts + align16(4ull * nb) / 4;
    uint32_t* dst = static_cast<uint32_t*>(d_dst);
    const T* src = static_cast<const T*>(d_src);
    sentinel_count_kernel<T><<<nb, kThreads, 0, s>>>(src, n, counts);
    sentinel_scan_kernel<<<1, 1024, 0, s>>>(counts, nb, static_cast<double>(n) * kMaxNonSentinels, dst, flag);
    sentinel_compact_kernel<T><<<nb, kThreads, 0, s>>>(src, n, counts, flag, dst);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

template <typename T>
void expand_t(const void* src, void* dst, size_t length) {
    const uint32_t* w = static_cast<const uint32_t*>(src);
    const uint32_t count = w[0];
    const char* values = reinterpret_cast<const char*>(w + 1);
    const uint32_t* idx = w + 1 + static_cast<size_t>(count) * (sizeof(T) / 4);
    std::memset(dst, 0, length);
    T* out = static_cast<T*>(dst);
    for (uint32_t k = 0; k < count; ++k) std::memcpy(&out[idx[k]], values + static_cast<size_t>(k) * sizeof(T), sizeof(T));
}

}  // namespace

extern "C" size_t pmb_sentinel_capacity_bytes(int type, size_t length) {
    const size_t es = elem_size(type);
    if (!es) return 0;
    // CheckSentinelCompression's bound (pmExecutionStub.cpp:3872-3873).
    const size_t mx = static_cast<size_t>((static_cast<double>(length) * kMaxNonSentinels + es - 1) / es) + 1;
    return sizeof(uint32_t) + mx * es + mx * sizeof(uint32_t);
}

extern "C" size_t pmb_sentinel_scratch_bytes(int type, size_t length) {
    const size_t es = elem_size(type);
    if (!es) return 0;
    return align16(4ull * num_blocks(length / es)) + 16;
}

extern "C" int pmb_sentinel_compress(int type, const void* d_src, size_t length, void* d_dst, size_t capacity,
                                     void* d_scratch, size_t scratch_bytes, void* stream) {
    const size_t es = elem_size(type);
    PMB_CHECK_ARG(es, "reduction data type %d outside [0,5]", type);
    PMB_CHECK_ARG(d_src && d_dst && d_scratch, "null pointer");
    PMB_CHECK_ARG(length % es == 0 && length / es < (size_t(1) << 32), "length %zu not a count of elements below 2^32",
                  length);
    PMB_CHECK_ARG(((reinterpret_cast<uintptr_t>(d_src) % es) | (reinterpret_cast<uintptr_t>(d_dst) & 3) |
                   (reinterpret_cast<uintptr_t>(d_scratch) & 15)) == 0,
                  "misaligned pointer");
    PMB_CHECK_ARG(capacity >= pmb_sentinel_capacity_bytes(type, length), "compressed buffer too small");
    PMB_CHECK_ARG(scratch_bytes >= pmb_sentinel_scratch_bytes(type, length), "scratch too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t n = length / es;
    if (n == 0) {
        PMB_CUDA_TRY(cudaMemsetAsync(d_dst, 0, sizeof(uint32_t), s));
        return PMB_SUCCESS;
    }
    switch (type) {
        case 0: return compress_t<int32_t>(d_src, n, d_dst, d_scratch, s);
        case 1: return compress_t<uint32_t>(d_src, n, d_dst, d_scratch, s);
        case 2: return compress_t<int64_t>(d_src, n, d_dst, d_scratch, s);
        case 3: return compress_t<uint64_t>(d_src, n, d_dst, d_scratch, s);
        case 4: return compress_t<float>(d_src, n, d_dst, d_scratch, s);
        default: return compress_t<double>(d_src, n, d_dst, d_scratch, s);
    }
}

extern "C" int pmb_sentinel_compressed(int type, size_t length, uint32_t count) {
    const size_t es = elem_size(type);
    return es && static_cast<double>(count) < static_cast<double>(length / es) * kMaxNonSentinels ? 1 : 0;
}

extern "C" int pmb_sentinel_expand(int type, const void* h_src, void* h_dst, size_t length) {
    const size_t es = elem_size(type);
    PMB_CHECK_ARG(es, "reduction data type %d outside [0,5]", type);
    PMB_CHECK_ARG(h_src && h_dst, "null pointer");
    PMB_CHECK_ARG(length % es == 0, "length %zu not a multiple of the element size", length);
    const uint32_t count = static_cast<const uint32_t*>(h_src)[0];
    PMB_CHECK_ARG(count <= length / es, "count %u above the element count", count);
    switch (es) {
        case 4: expand_t<uint32_t>(h_src, h_dst, length); break;
        default: expand_t<uint64_t>(h_src, h_dst, length); break;
    }
    return PMB_SUCCESS;
}
