// radixSort subtask kernels: stable LSD radix sort of uint32 keys.
//
// Semantics: each pass is one stable counting-sort round on a digit
// (testSuite/radixSort/source/code/src/radixSort.cpp:55-69
// serialRadixSortRound).  In the reference, a round runs per subtask and the
// redistribution callback (:150-162) then concatenates the per-subtask digit
// buckets in order (digit major, subtask minor), which is exactly one global
// stable counting sort on that digit -- what a pass here computes in one go.
// The reference uses 4-bit digits (radixSort.h:42-46); 8-bit digits need half
// the passes over HBM for the same sorted result.
//
// Design (onesweep): one histogram kernel reads the keys once and counts the
// digits of every pass.  Each pass is then a single launch: a 256-thread CTA
// takes the next 4096-key tile from a global counter, ranks its keys stably
// with warp-level ballots/popc (warp-striped order), publishes its per-digit
// counts, and thread d looks back over predecessor tiles' status words for
// digit d to get the tile's global offset for that digit.  Keys are reordered
// by digit in shared memory, then written so that each digit run is a
// contiguous, coalesced store.  Per pass: 4 bytes read + 4 bytes written per
// key, plus the small status array.
#include "lookback.cuh"
#include "pmb_common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096 keys
constexpr size_t kHeaderBytes = 256;      // hdr[1] = error word, hdr[2+p] = tile counter of pass p
constexpr size_t kHistBytes = 4096;       // [passes][radix] u32, passes*radix <= 1024
constexpr uint32_t kCountMask = (1u << 30) - 1;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr int kLook = 4;                  // predecessor tiles read per look-back round

template <int BITS>
__global__ void __launch_bounds__(kThreads)
radix_hist_kernel(const uint32_t* __restrict__ keys, size_t n, int begin_bit, int passes,
                  uint32_t* __restrict__ hist) {
    constexpr int RADIX = 1 << BITS;
    constexpr uint32_t MASK = RADIX - 1;
    __shared__ uint32_t sh[1024];
    const int total = passes * RADIX;
    for (int i = threadIdx.x; i < total; i += kThreads) sh[i] = 0;
    __syncthreads();
    const size_t nq = n / 4;
    const uint4* q = reinterpret_cast<const uint4*>(keys);
    for (size_t i = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < nq;
         i += static_cast<size_t>(gridDim.x) * kThreads) {
        const uint4 v = __ldg(q + i);
        const uint32_t k4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j)
            for (int p = 0; p < passes; ++p)
                atomicAdd(&sh[p * RADIX + ((k4[j] >> (begin_bit + p * BITS)) & MASK)], 1u);
    }
    if (blockIdx.x == 0) {
        for (size_t i = nq * 4 + threadIdx.x; i < n; i += kThreads)
            for (int p = 0; p < passes; ++p)
                atomicAdd(&sh[p * RADIX + ((keys[i] >> (begin_bit + p * BITS)) & MASK)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < total; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Exclusive scan of one value per thread across the CTA (values of threads >=
// `count` must be 0).  Returns the exclusive prefix of the calling thread.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* s_tmp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t inc = pmb::warp_inclusive_scan_u32(x, lane);
    if (lane == 31) s_tmp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < kWarps ? s_tmp[lane] : 0u;
        const uint32_t wi = pmb::warp_inclusive_scan_u32(w, lane);
        if (lane < kWarps) s_tmp[lane] = wi - w;
    }
    __syncthreads();
    const uint32_t r = s_tmp[warp] + inc - x;
    __syncthreads();
    return r;
}

template <int BITS, bool VALUES>
__global__ void __launch_bounds__(kThreads, VALUES ? 3 : 4)
onesweep_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, const uint32_t* __restrict__ vin,
                uint32_t* __restrict__ vout, size_t n, int shift, const uint32_t* __restrict__ hist_pass,
                uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ err, uint32_t* __restrict__ status) {
    constexpr int RADIX = 1 << BITS;
    constexpr uint32_t MASK = RADIX - 1;
    static_assert(RADIX <= kThreads, "one digit per thread");
    __shared__ __align__(16) uint32_t s_keys[kTile];
    __shared__ uint32_t s_vals[VALUES ? kTile : 1];
    __shared__ __align__(16) uint32_t s_whist[kWarps][RADIX];
    __shared__ uint32_t s_dummy[kWarps][32];
    __shared__ uint32_t s_mdummy[kWarps][32];
    // Per warp and digit, the lanes holding it (two items in turn); used only
    // while ranking, so it shares its storage with s_keys.
    static_assert(2 * kWarps * RADIX <= kTile, "match words fit in the key buffer");
    auto s_match = reinterpret_cast<uint32_t (*)[kWarps][RADIX]>(s_keys);
    __shared__ uint32_t s_goff[RADIX];
    __shared__ uint32_t s_tmp[kWarps];
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    {
        static_assert((kWarps * RADIX) % 4 == 0, "16-byte clears");
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (int i = tid; i < kWarps * RADIX / 4; i += kThreads) reinterpret_cast<uint4*>(&s_whist[0][0])[i] = z;
        for (int i = tid; i < 2 * kWarps * RADIX / 4; i += kThreads) reinterpret_cast<uint4*>(&s_match[0][0][0])[i] = z;
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t wbase = static_cast<size_t>(tile) * kTile + static_cast<size_t>(warp) * (kItems * 32);

    uint32_t key[kItems];
    uint32_t rank[kItems];
    // Every tile but the last is full: its loads, ranks, scatter and stores run
    // without per-key bounds tests (branches are what limits this kernel).
    const bool full = static_cast<size_t>(tile + 1) * kTile <= n;
    if (full) {
#pragma unroll
        for (int i = 0; i < kItems; ++i) key[i] = in[wbase + i * 32 + lane];
    } else {
#pragma unroll
        for (int i = 0; i < kItems; ++i) {
            const size_t idx = wbase + i * 32 + lane;
            key[i] = idx < n ? in[idx] : 0u;
        }
    }
    // Stable warp-level ranking in (warp, item, lane) order.  Every lane ORs
    // its bit into the word of its digit (shared-memory atomic OR: the order
    // of the lanes does not matter), and reads back the set of lanes holding
    // the same digit.  The lowest of them (the leader) advances the warp's
    // running count for that digit and, one item later, clears the word;
    // consecutive items use alternate word sets, so a clear is ordered before
    // the word's next use by the syncs in between.  Invalid lanes of a ragged
    // last tile, and lanes that are not leaders, do the same loads and stores
    // on private dummy words: no divergent branch.
    uint32_t* prev_clear = &s_mdummy[warp][lane];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const bool valid = full || wbase + i * 32 + lane < n;
        const uint32_t d = (key[i] >> shift) & MASK;
        uint32_t* mw = valid ? &s_match[i & 1][warp][d] : &s_mdummy[warp][lane];
        atomicOr(mw, 1u << lane);
        __syncwarp();
        const uint32_t peers = valid ? *mw : (1u << lane);
        *prev_clear = 0;  // the previous item's word, if this lane led it
        const int leader = __ffs(peers) - 1;
        const bool lead = valid && lane == leader;
        uint32_t* slot = lead ? &s_whist[warp][d] : &s_dummy[warp][lane];
        const uint32_t cnt = atomicAdd(slot, static_cast<uint32_t>(__popc(peers)));
        prev_clear = lead ? mw : &s_mdummy[warp][lane];
        __syncwarp();
        rank[i] = __shfl_sync(0xffffffffu, cnt, leader) + __popc(peers & pmb::lanemask_lt());
    }
    *prev_clear = 0;
    __syncthreads();

    // Per digit: warp offsets within the tile and the tile's digit count.
    uint32_t my_cnt = 0;
    if (tid < RADIX) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t t = s_whist[w][tid];
            s_whist[w][tid] = my_cnt;
            my_cnt += t;
        }
        pmb::st_relaxed_u32(&status[static_cast<size_t>(tile) * RADIX + tid],
                            (tile == 0 ? kFlagInc : kFlagAgg) | my_cnt);
    }
    const uint32_t tile_start = block_exclusive_scan(tid < RADIX ? my_cnt : 0u, s_tmp);
    const uint32_t digit_base = block_exclusive_scan(tid < RADIX ? hist_pass[tid] : 0u, s_tmp);

    if (tid < RADIX) {
        // One table per lookup below: each is a shared load at a data-dependent
        // (bank-conflicting) address, so the offsets are pre-added.
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s_whist[w][tid] += tile_start;
        uint32_t excl = 0;
        if (tile > 0) {
            // kLook predecessors per round, loaded together; only those nearer
            // than the nearest inclusive count must be ready.
            bool gave_up = false;
            for (long long t0 = static_cast<long long>(tile) - 1; t0 >= 0 && !gave_up; t0 -= kLook) {
                uint32_t s[kLook];
#pragma unroll
                for (int j = 0; j < kLook; ++j)
                    s[j] = t0 - j >= 0 ? pmb::ld_relaxed_u32(&status[static_cast<size_t>(t0 - j) * RADIX + tid])
                                       : kFlagInc;
                uint32_t polls = 0;
                int first;
                for (;;) {
                    first = kLook;
#pragma unroll
                    for (int j = kLook - 1; j >= 0; --j)
                        if ((s[j] >> 30) == 2) first = j;
                    bool pending = false;
#pragma unroll
                    for (int j = 0; j < kLook; ++j) pending |= j < first && (s[j] >> 30) == 0;
                    if (!pending) break;
                    if (++polls > pmb::kSpinLimit) {
                        gave_up = true;
                        break;
                    }
                    __nanosleep(64);
#pragma unroll
                    for (int j = 0; j < kLook; ++j)
                        if (j < first && (s[j] >> 30) == 0)
                            s[j] = pmb::ld_relaxed_u32(&status[static_cast<size_t>(t0 - j) * RADIX + tid]);
                }
#pragma unroll
                for (int j = 0; j < kLook; ++j)
                    if (j <= first) excl += s[j] & kCountMask;
                if (first < kLook) break;
            }
            if (gave_up) atomicOr(err, pmb::kErrLookbackTimeout);
            pmb::st_relaxed_u32(&status[static_cast<size_t>(tile) * RADIX + tid],
                                kFlagInc | ((excl + my_cnt) & kCountMask));
        }
        s_goff[tid] = digit_base + excl - tile_start;  // output index = s_goff[d] + tile position
    }
    __syncthreads();

#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (full || wbase + i * 32 + lane < n) {
            const uint32_t d = (key[i] >> shift) & MASK;
            const uint32_t pos = s_whist[warp][d] + rank[i];
            s_keys[pos] = key[i];
            if constexpr (VALUES) s_vals[pos] = vin[wbase + i * 32 + lane];
        }
    }
    __syncthreads();
    const size_t tbase = static_cast<size_t>(tile) * kTile;
    if (full) {
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const int p = tid + j * kThreads;
            const uint32_t k = s_keys[p];
            const uint32_t d = (k >> shift) & MASK;
            const uint32_t g = s_goff[d] + p;
            out[g] = k;
            if constexpr (VALUES) vout[g] = s_vals[p];
        }
    } else {
        const int tile_n = static_cast<int>(n - tbase);
        for (int p = tid; p < tile_n; p += kThreads) {
            const uint32_t k = s_keys[p];
            const uint32_t d = (k >> shift) & MASK;
            const uint32_t g = s_goff[d] + p;
            out[g] = k;
            if constexpr (VALUES) vout[g] = s_vals[p];
        }
    }
}

size_t num_tiles(size_t n) { return (n + kTile - 1) / kTile; }

size_t scratch_bytes_for(size_t n, int bits) {
    return kHeaderBytes + kHistBytes + 4 * num_tiles(n) * (static_cast<size_t>(1) << bits);
}

template <int BITS>
int sort_t(uint32_t* keys, uint32_t* alt, uint32_t* vals, uint32_t* valt, size_t n, int begin_bit, int passes,
           void* scratch, cudaStream_t s) {
    constexpr int RADIX = 1 << BITS;
    char* base = static_cast<char*>(scratch);
    uint32_t* hdr = reinterpret_cast<uint32_t*>(base);
    uint32_t* hist = reinterpret_cast<uint32_t*>(base + kHeaderBytes);
    uint32_t* status = reinterpret_cast<uint32_t*>(base + kHeaderBytes + kHistBytes);
    const size_t tiles = num_tiles(n);
    PMB_CUDA_TRY(cudaMemsetAsync(base, 0, kHeaderBytes + kHistBytes, s));
    int dev = 0, sms = 148;
    PMB_CUDA_TRY(cudaGetDevice(&dev));
    PMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t want = (n / 4 + kThreads - 1) / kThreads;
    const unsigned hgrid = static_cast<unsigned>(want < static_cast<size_t>(sms) * 8 ? (want ? want : 1) : sms * 8);
    radix_hist_kernel<BITS><<<hgrid, kThreads, 0, s>>>(keys, n, begin_bit, passes, hist);
    PMB_CUDA_TRY(cudaGetLastError());
    const uint32_t* src = keys;
    uint32_t* dst = alt;
    const uint32_t* vsrc = vals;
    uint32_t* vdst = valt;
    for (int p = 0; p < passes; ++p) {
        PMB_CUDA_TRY(cudaMemsetAsync(status, 0, 4 * tiles * RADIX, s));
        if (vals)
            onesweep_kernel<BITS, true><<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(
                src, dst, vsrc, vdst, n, begin_bit + p * BITS, hist + p * RADIX, &hdr[2 + p], &hdr[1], status);
        else
            onesweep_kernel<BITS, false><<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(
                src, dst, nullptr, nullptr, n, begin_bit + p * BITS, hist + p * RADIX, &hdr[2 + p], &hdr[1], status);
        PMB_CUDA_TRY(cudaGetLastError());
        src = dst;
        dst = (dst == alt) ? keys : alt;
        if (vals) {
            vsrc = vdst;
            vdst = (vdst == valt) ? vals : valt;
        }
    }
    if (src != keys) {
        PMB_CUDA_TRY(cudaMemcpyAsync(keys, src, 4 * n, cudaMemcpyDeviceToDevice, s));
        if (vals) PMB_CUDA_TRY(cudaMemcpyAsync(vals, vsrc, 4 * n, cudaMemcpyDeviceToDevice, s));
    }
    return PMB_SUCCESS;
}

int sort_checked(uint32_t* keys, uint32_t* alt, uint32_t* vals, uint32_t* valt, size_t n, int begin_bit, int end_bit,
                 int bits, void* scratch, size_t scratch_bytes, cudaStream_t s) {
    if (n == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(keys && alt && scratch, "null pointer");
    PMB_CHECK_ARG(keys != alt, "keys and alternate buffer must differ");
    PMB_CHECK_ARG((vals == nullptr) == (valt == nullptr), "values need both buffers");
    PMB_CHECK_ARG(vals == nullptr || (vals != valt && vals != keys && vals != alt && valt != keys && valt != alt),
                  "value buffers must be distinct from each other and from the key buffers");
    PMB_CHECK_ARG(bits == 4 || bits == 8, "digit width %d not 4 or 8", bits);
    PMB_CHECK_ARG(0 <= begin_bit && begin_bit < end_bit && end_bit <= 32 && (end_bit - begin_bit) % bits == 0,
                  "bit range [%d,%d) not a multiple of %d-bit digits", begin_bit, end_bit, bits);
    PMB_CHECK_ARG(n < (1ull << 30), "sort length %zu not below 2^30", n);
    PMB_CHECK_ARG(((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(scratch)) & 15) == 0,
                  "keys and scratch must be 16-byte aligned");
    const size_t need = scratch_bytes_for(n, bits);
    if (scratch_bytes < need)
        return pmb::fail(PMB_BEYOND_LIMITS, "radix scratch %zu bytes, need %zu", scratch_bytes, need);
    const int passes = (end_bit - begin_bit) / bits;
    return bits == 8 ? sort_t<8>(keys, alt, vals, valt, n, begin_bit, passes, scratch, s)
                     : sort_t<4>(keys, alt, vals, valt, n, begin_bit, passes, scratch, s);
}

}  // namespace

extern "C" size_t pmb_radix_sort_scratch_bytes(size_t n, int bits_per_pass) {
    return scratch_bytes_for(n, bits_per_pass == 4 ? 4 : 8);
}

extern "C" int pmb_radix_sort_u32(uint32_t* d_keys, uint32_t* d_alt, size_t n, int begin_bit, int end_bit,
                                  int bits_per_pass, void* d_scratch, size_t scratch_bytes, void* stream) {
    return sort_checked(d_keys, d_alt, nullptr, nullptr, n, begin_bit, end_bit, bits_per_pass, d_scratch,
                        scratch_bytes, static_cast<cudaStream_t>(stream));
}

extern "C" int pmb_radix_sort_pairs_u32(uint32_t* d_keys, uint32_t* d_alt, uint32_t* d_vals, uint32_t* d_vals_alt,
                                        size_t n, int begin_bit, int end_bit, int bits_per_pass, void* d_scratch,
                                        size_t scratch_bytes, void* stream) {
    PMB_CHECK_ARG(d_vals && d_vals_alt, "null value buffer");
    return sort_checked(d_keys, d_alt, d_vals, d_vals_alt, n, begin_bit, end_bit, bits_per_pass, d_scratch,
                        scratch_bytes, static_cast<cudaStream_t>(stream));
}

// Digit counts of the first pass of the last sort run with `d_scratch`
// (uint32 per digit, 2^bits of them), copied on the stream into d_counts:
// the per-subtask bins the reference's radixSort round hands to its
// redistribution callback (radixSort.cpp:127-148).
extern "C" int pmb_radix_sort_histogram(const void* d_scratch, int bits_per_pass, void* d_counts, void* stream) {
    PMB_CHECK_ARG(d_scratch && d_counts, "null pointer");
    PMB_CHECK_ARG(bits_per_pass == 4 || bits_per_pass == 8, "digit width %d not 4 or 8", bits_per_pass);
    PMB_CUDA_TRY(cudaMemcpyAsync(d_counts, static_cast<const char*>(d_scratch) + kHeaderBytes,
                                 sizeof(uint32_t) << bits_per_pass, cudaMemcpyDeviceToDevice,
                                 static_cast<cudaStream_t>(stream)));
    return PMB_SUCCESS;
}
