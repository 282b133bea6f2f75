// matrixMultiply / luDecomposition GEMM for sm_100a: fp32 in, fp32 out,
// computed as a BF16x3 split-precision product on the 5th-generation tensor
// cores (tcgen05) with FP32 accumulation in tensor memory.
//
// Semantics (row-major): C = alpha * A * B + beta * C, A: M x K (lda),
// B: K x N (ldb), C: M x N (ldc).  The reference reaches this through
// cublasSgemm (testSuite/matrixMultiplyBlas/source/code/src/
// matrixMultiplyBlasCUDA.cu:54-77, luDecompositionCUDA.cu:153-193) and
// cblas_sgemm on the CPU (matrixMultiplyBlas.cpp:62-65).
//
// Split precision: x = hi + lo with hi = bf16(x) and lo = bf16(x - hi), so
// A*B ~= Ahi*Bhi + Ahi*Blo + Alo*Bhi (the Alo*Blo term, ~2^-18 relative, is
// dropped).  All three products accumulate into the same FP32 TMEM tile.
//
// Accumulation: the tensor core's FP32 accumulate is not round-to-nearest, so
// its error grows with the number of MMA results added into one accumulator
// (measured: ~2.8e-5 normwise at K = 8192 in a single accumulator).  The K
// loop is therefore cut into segments of 1024: each segment accumulates into
// one of two 256-column TMEM buffers, and the epilogue warps drain a finished
// buffer into C in IEEE FP32 (C = alpha*P + beta*C for the first segment,
// C += alpha*P after) while the MMAs continue in the other buffer.
//
// Design: a split pass writes Ahi/Alo (M x Kp) and the transposed Bhi/Blo
// (N x Kp) as K-major bf16.  The GEMM kernel owns a 128 x 256 output tile per
// CTA and runs three warp roles:
//   warp 0    TMA producer: one thread streams 32-deep K slices of the four
//             operand tiles into a 4-stage shared-memory ring (SWIZZLE_64B),
//             arming each stage's mbarrier with the expected byte count;
//   warp 1    allocates 512 TMEM columns, then one thread issues the
//             tcgen05.mma instructions (M=128, N=256, K=16, 3 per K step),
//             frees each stage back to the producer with tcgen05.commit and
//             signals each finished accumulator segment;
//   warps 2-5 epilogue: tcgen05.ld each segment (one row per thread), apply
//             alpha/beta and accumulate into C, then hand the buffer back.
// Products with K <= 64 (one K slice: the LU trailing update) take a third
// kernel that moves C through shared memory by TMA (gemm_update_2sm_kernel).
// Every mbarrier wait is bounded: on expiry the kernel records an error in the
// workspace header, skips the remaining work, waits (bounded) for its own
// in-flight tensor-core work and frees its TMEM before returning.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pmb_common.cuh"

namespace {

constexpr int BM = 128, BN = 256, BK = 32;  // BK in bf16 elements (64 bytes: one SWIZZLE_64B row)
constexpr int kStages = 4;
constexpr int kThreads = 192;
constexpr int kTileA = BM * BK * 2;   // 8 KB
constexpr int kTileB = BN * BK * 2;   // 16 KB
constexpr int kStageBytes = 2 * kTileA + 2 * kTileB;  // 48 KB
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align slack*/ + 256 /*barriers*/;
constexpr uint32_t kTmemCols = 512;         // two 256-column accumulators
constexpr int kFlushStages = 32;            // K = 1024 per accumulator segment
constexpr uint32_t kWaitLimit = 1u << 21;   // try_wait polls (each suspends <= ~1 us)
constexpr uint32_t kErrTimeout = 4;         // workspace error bit

// Instruction descriptor, kind::f16: F32 accumulator, BF16 A and B, both
// K-major, N = 256, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor for a K-major SWIZZLE_64B tile: rows of 64
// bytes, 8-row core groups 512 bytes apart.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFF);
    d |= static_cast<uint64_t>(1) << 16;                 // leading byte offset (unused for swizzled K-major)
    d |= static_cast<uint64_t>(512 >> 4) << 32;          // stride byte offset: 8 rows x 64 B
    d |= static_cast<uint64_t>(1) << 46;                 // descriptor version (sm_100)
    d |= static_cast<uint64_t>(4) << 61;                 // SWIZZLE_64B
    return d;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Bounded wait for the phase with the given parity; false on expiry.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
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

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct GemmMaps {
    CUtensorMap ah, al, bh, bl;
};

__global__ void __launch_bounds__(kThreads, 1)
gemm_bf16x3_kernel(const __grid_constant__ GemmMaps maps, int M, int N, int KT, float alpha, float beta,
                   float* __restrict__ C, int64_t ldc, uint32_t* __restrict__ err) {
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the split pass launched before it
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    // bars[0..S): stage full, [S..2S): stage empty, [2S, 2S+2): accumulator b
    // full, [2S+2, 2S+4): accumulator b drained, [2S+4]: teardown
    uint64_t* acc_full = bars + 2 * kStages;
    uint64_t* acc_empty = bars + 2 * kStages + 2;
    uint64_t* teardown = bars + 2 * kStages + 4;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 5);
    __shared__ volatile int s_fail;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;

    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&bars[s]), 1);
            mbar_init(smem_u32(&bars[kStages + s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 4);  // one arrival per epilogue warp
        }
        mbar_init(smem_u32(teardown), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---- producer ----
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % kStages;
            if (kt >= kStages && !mbar_wait(smem_u32(&bars[kStages + s]), ((kt / kStages) + 1) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            if (s_fail) break;
            uint8_t* st = smem + s * kStageBytes;
            const uint32_t full = smem_u32(&bars[s]);
            mbar_expect_tx(full, kStageBytes);
            const int k = kt * BK;
            tma_load_2d(smem_u32(st), &maps.ah, k, m0, full);
            tma_load_2d(smem_u32(st + kTileA), &maps.al, k, m0, full);
            tma_load_2d(smem_u32(st + 2 * kTileA), &maps.bh, k, n0, full);
            tma_load_2d(smem_u32(st + 2 * kTileA + kTileB), &maps.bl, k, n0, full);
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer ----
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % kStages;
            const int seg = kt / kFlushStages, seg_k = kt % kFlushStages, b = seg & 1;
            if (seg_k == 0 && seg >= 2 && !mbar_wait(smem_u32(&acc_empty[b]), ((seg >> 1) - 1) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            if (!mbar_wait(smem_u32(&bars[s]), (kt / kStages) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc = tmem + 256u * b;
            const uint32_t st = smem_u32(smem + s * kStageBytes);
            const uint32_t a_hi = st, a_lo = st + kTileA, b_hi = st + 2 * kTileA, b_lo = st + 2 * kTileA + kTileB;
#pragma unroll
            for (int k16 = 0; k16 < BK / 16; ++k16) {
                const uint32_t off = k16 * 32;  // 16 bf16 = 32 bytes along the swizzled row
                umma_bf16(acc, umma_desc_sw64(a_hi + off), umma_desc_sw64(b_hi + off), (seg_k | k16) != 0);
                umma_bf16(acc, umma_desc_sw64(a_hi + off), umma_desc_sw64(b_lo + off), 1u);
                umma_bf16(acc, umma_desc_sw64(a_lo + off), umma_desc_sw64(b_hi + off), 1u);
            }
            umma_commit(smem_u32(&bars[kStages + s]));
            if (seg_k == kFlushStages - 1 || kt == KT - 1) umma_commit(smem_u32(&acc_full[b]));
        }
    } else if (warp >= 2) {
        // ---- epilogue: drain each accumulator segment into C ----
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int row = m0 + 32 * q + lane;
        const int nseg = (KT + kFlushStages - 1) / kFlushStages;
        for (int seg = 0; seg < nseg; ++seg) {
            const int b = seg & 1;
            if (!mbar_wait(smem_u32(&acc_full[b]), (seg >> 1) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            if (s_fail) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const float bscale = seg == 0 ? beta : 1.0f;
#pragma unroll 1
            for (int c = 0; c < BN / 16; ++c) {
                uint32_t r[16];
                tmem_ld16(tmem + 256u * b + (static_cast<uint32_t>(32 * q) << 16) + 16 * c, r);
                const int col = n0 + 16 * c;
                if (row >= M || col >= N) continue;
                float* crow = C + static_cast<int64_t>(row) * ldc + col;
                const bool vec = col + 16 <= N && ((reinterpret_cast<uintptr_t>(crow) & 15) == 0);
                if (vec) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4) {
                        float4 o;
                        o.x = alpha * __uint_as_float(r[j]);
                        o.y = alpha * __uint_as_float(r[j + 1]);
                        o.z = alpha * __uint_as_float(r[j + 2]);
                        o.w = alpha * __uint_as_float(r[j + 3]);
                        if (bscale != 0.0f) {
                            const float4 old = *reinterpret_cast<const float4*>(crow + j);
                            o.x += bscale * old.x;
                            o.y += bscale * old.y;
                            o.z += bscale * old.z;
                            o.w += bscale * old.w;
                        }
                        *reinterpret_cast<float4*>(crow + j) = o;
                    }
                } else {
                    for (int j = 0; j < 16 && col + j < N; ++j) {
                        float o = alpha * __uint_as_float(r[j]);
                        if (bscale != 0.0f) o += bscale * crow[j];
                        crow[j] = o;
                    }
                }
            }
            // Buffer b is drained: its tcgen05.ld have completed (tmem_ld16 waits).
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[b])) : "memory");
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (s_fail && lane == 0) {
            // Make sure every MMA this CTA issued has retired before freeing TMEM.
            umma_commit(smem_u32(teardown));
            mbar_wait(smem_u32(teardown), 0);
        }
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// ---- 2-SM kernel: one 256 x 256 output tile per CTA pair ----------------------
// A cluster of two CTAs on two SMs issues tcgen05.mma.cta_group::2 with M = 256,
// N = 256: each CTA stages its own 128 rows of A and its own 128 rows of B^T
// (non-multicast TMA), the leader CTA's single MMA thread reads both CTAs'
// shared memory, and each CTA's tensor memory receives its 128 rows of the
// tile.  Per CTA and K-slice that is 64 KB of operands for the work the 1-SM
// kernel needs 96 KB for, and the 128-byte K slices (SWIZZLE_128B) halve the
// number of TMA requests; three stages fill the shared memory.  Products with
// few tiles use N = 128 per pair instead (Pair2<128>: twice the pairs busy,
// four 48 KB stages).
//   full[s]     leader only: one arrive.expect_tx from each CTA's producer plus
//               both CTAs' TMA bytes (the peer's loads signal it remotely);
//   empty[s]    both CTAs: multicast tcgen05.commit from the leader;
//   acc_full[b] both CTAs: multicast commit after a 1024-deep K segment;
//   acc_empty[b] leader only: one remote arrive per epilogue warp of each CTA.
// The epilogue stages each 32 x 16 chunk through shared memory so that global
// reads and writes of C are whole 64-byte row pieces.
constexpr int BK2 = 64;                                   // 128-byte rows
constexpr int kStages2 = 3;
constexpr int kHalf2 = 128 * BK2 * 2;                     // 16 KB: 128 rows of one operand
constexpr int kStage2Bytes = 4 * kHalf2;                  // A hi, A lo, B hi, B lo halves
constexpr int kStageOutFloats = 4 * 32 * 20;              // per-warp 32 x 16 staging, row stride 20
constexpr int kSmem2Bytes = kStages2 * kStage2Bytes + kStageOutFloats * 4 + 1024 + 256;

// Tile shape of the pair kernel: 256 x TN outputs per CTA pair (TN = 256, or
// 128 when a product has too few 256 x 256 tiles to occupy the SM pairs).
// Each CTA stages TN/2 rows of B^T; 192 KB of stages either way (3 x 64 KB or
// 4 x 48 KB); two TN-column accumulators in tensor memory.
template <int TN>
struct Pair2 {
    static_assert(TN == 256 || TN == 128, "pair tile width");
    static constexpr int kBHalf = (TN / 2) * BK2 * 2;
    static constexpr int kStageBytes = 2 * kHalf2 + 2 * kBHalf;
    static constexpr int kStages = TN == 256 ? 3 : 4;
    static constexpr int kSmemBytes = kStages * kStageBytes + kStageOutFloats * 4 + 1024 + 256;
    static constexpr uint32_t kTmemCols = 2 * TN;
    static constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                                       ((uint32_t)(256 >> 4) << 24);
};
static_assert(Pair2<256>::kSmemBytes == kSmem2Bytes && Pair2<128>::kSmemBytes <= kSmem2Bytes, "pair shared memory");
constexpr int kFlush2 = 16;                               // K = 1024 per accumulator segment
constexpr int kGroupRows = 8;                             // tile rows per raster group
// K-major SWIZZLE_128B tile: rows of 128 bytes, 8-row core groups 1024 bytes apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFF);
    d |= static_cast<uint64_t>(1) << 16;
    d |= static_cast<uint64_t>(1024 >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(2) << 61;  // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(uint32_t saddr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx_cluster(uint32_t cbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cluster.shared::cluster.b64 _, [%0], %1;" ::"r"(cbar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cbar) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cbar) : "memory");
}
// TMA load into this CTA's shared memory, completion on an mbarrier of either CTA of the pair.
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t cbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.cta_group::2 [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(cbar)
        : "memory");
}
__device__ __forceinline__ void umma_bf16_pair_i(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                                 uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive once on the mbarrier at this shared offset in both CTAs of the pair.
__device__ __forceinline__ void umma_commit_pair(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
        "h"(static_cast<uint16_t>(3))
        : "memory");
}

// Grouped tile order of the 2-SM kernels: CTA pair blockIdx.x / 2 -> 256 x tn
// tile (pm, pn).  Consecutive pairs sweep the columns of a band of kGroupRows
// tile rows.
__device__ __forceinline__ void pair_tile(int M, int N, int tn, int pid, int& pm, int& pn) {
    const int num_pm = (M + 255) / 256, num_pn = (N + tn - 1) / tn;
    const int per_group = kGroupRows * num_pn;
    const int first = (pid / per_group) * kGroupRows;
    const int rows = min(num_pm - first, kGroupRows);
    const int in_group = pid % per_group;
    pm = first + in_group % rows;
    pn = in_group / rows;
}

// One 256 x TN tile of one product, computed by a CTA pair: `pid` is the
// pair's tile index within the product.  `maps` must live in the parameter
// (or global) space: its address goes to the TMA loads.
template <int TN>
__device__ __forceinline__ void gemm2_tile(const GemmMaps& maps, int M, int N, int KT, float alpha, float beta,
                                           float* __restrict__ C, int64_t ldc, uint32_t* __restrict__ err, int pid) {
    using P = Pair2<TN>;
    constexpr int kStages2 = P::kStages, kStage2Bytes = P::kStageBytes, kBHalf = P::kBHalf;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float* stage_out = reinterpret_cast<float*>(smem + kStages2 * kStage2Bytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages2 * kStage2Bytes + kStageOutFloats * 4);
    uint64_t* full = bars;                          // [kStages2]
    uint64_t* empty = bars + kStages2;              // [kStages2]
    uint64_t* acc_full = bars + 2 * kStages2;       // [2]
    uint64_t* acc_empty = bars + 2 * kStages2 + 2;  // [2]
    uint64_t* teardown = bars + 2 * kStages2 + 4;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages2 + 5);
    __shared__ volatile int s_fail;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    // Grouped tile order: consecutive pairs sweep the columns of a band of
    // kGroupRows tile rows, so the pairs resident at one time share A and B
    // panels (read once from HBM, then from L2) instead of each wave reading
    // every row panel of A.
    int pm, pn;
    pair_tile(M, N, TN, pid, pm, pn);
    const int m0 = pm * 256 + 128 * static_cast<int>(rank);     // this CTA's rows of A and C
    const int n0 = pn * TN;                                     // the pair's columns
    const int nb0 = n0 + (TN / 2) * static_cast<int>(rank);     // this CTA's rows of B^T

    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int s = 0; s < kStages2; ++s) {
            mbar_init(smem_u32(&full[s]), 2);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 8);  // 4 epilogue warps in each CTA
        }
        mbar_init(smem_u32(teardown), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(P::kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    cluster_sync_all();  // the peer's barriers exist before anyone signals them
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---- producer (both CTAs) ----
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % kStages2;
            if (kt >= kStages2 && !mbar_wait(smem_u32(&empty[s]), ((kt / kStages2) + 1) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            if (s_fail) break;
            uint8_t* st = smem + s * kStage2Bytes;
            const uint32_t fbar = cluster_addr(smem_u32(&full[s]), 0);
            mbar_arrive_expect_tx_cluster(fbar, kStage2Bytes);
            const int k = kt * BK2;
            tma_load_2d_pair(smem_u32(st), &maps.ah, k, m0, fbar);
            tma_load_2d_pair(smem_u32(st + kHalf2), &maps.al, k, m0, fbar);
            tma_load_2d_pair(smem_u32(st + 2 * kHalf2), &maps.bh, k, nb0, fbar);
            tma_load_2d_pair(smem_u32(st + 2 * kHalf2 + kBHalf), &maps.bl, k, nb0, fbar);
        }
    } else if (warp == 1 && lane == 0 && rank == 0) {
        // ---- MMA issuer (leader CTA) ----
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % kStages2;
            const int seg = kt / kFlush2, seg_k = kt % kFlush2, b = seg & 1;
            if (seg_k == 0 && seg >= 2 && !mbar_wait(smem_u32(&acc_empty[b]), ((seg >> 1) - 1) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            if (!mbar_wait(smem_u32(&full[s]), (kt / kStages2) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc = tmem + static_cast<uint32_t>(TN) * b;
            const uint32_t st = smem_u32(smem + s * kStage2Bytes);
            const uint32_t a_hi = st, a_lo = st + kHalf2, b_hi = st + 2 * kHalf2, b_lo = st + 2 * kHalf2 + kBHalf;
#pragma unroll
            for (int k16 = 0; k16 < BK2 / 16; ++k16) {
                const uint32_t off = k16 * 32;  // 16 bf16 = 32 bytes along the swizzled row
                umma_bf16_pair_i(acc, umma_desc_sw128(a_hi + off), umma_desc_sw128(b_hi + off), P::kIdesc,
                                 (seg_k | k16) != 0);
                umma_bf16_pair_i(acc, umma_desc_sw128(a_hi + off), umma_desc_sw128(b_lo + off), P::kIdesc, 1u);
                umma_bf16_pair_i(acc, umma_desc_sw128(a_lo + off), umma_desc_sw128(b_hi + off), P::kIdesc, 1u);
            }
            umma_commit_pair(smem_u32(&empty[s]));
            if (seg_k == kFlush2 - 1 || kt == KT - 1) umma_commit_pair(smem_u32(&acc_full[b]));
        }
    } else if (warp >= 2) {
        // ---- epilogue (both CTAs): drain each segment of this CTA's 128 rows ----
        const int q = warp & 3;
        float* stg = stage_out + q * 32 * 20;
        const int nseg = (KT + kFlush2 - 1) / kFlush2;
        const bool vec_ok = (ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0;
        for (int seg = 0; seg < nseg; ++seg) {
            const int b = seg & 1;
            if (!mbar_wait(smem_u32(&acc_full[b]), (seg >> 1) & 1)) {
                s_fail = 1;
                atomicOr(err, kErrTimeout);
                break;
            }
            if (s_fail) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const float bscale = seg == 0 ? beta : 1.0f;
#pragma unroll 1
            for (int c = 0; c < TN / 16; ++c) {
                uint32_t r[16];
                tmem_ld16(tmem + static_cast<uint32_t>(TN) * b + (static_cast<uint32_t>(32 * q) << 16) + 16 * c, r);
                float4* mine = reinterpret_cast<float4*>(stg + lane * 20);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mine[j] = make_float4(__uint_as_float(r[4 * j]), __uint_as_float(r[4 * j + 1]),
                                          __uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]));
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int rl = i * 8 + (lane >> 2), c4 = (lane & 3) * 4;
                    const int grow = m0 + 32 * q + rl, gcol = n0 + 16 * c + c4;
                    if (grow >= M || gcol >= N) continue;
                    float4 v = *reinterpret_cast<const float4*>(stg + rl * 20 + c4);
                    float* cp = C + static_cast<int64_t>(grow) * ldc + gcol;
                    if (vec_ok && gcol + 4 <= N) {
                        float4 o = make_float4(alpha * v.x, alpha * v.y, alpha * v.z, alpha * v.w);
                        if (bscale != 0.0f) {
                            const float4 old = *reinterpret_cast<const float4*>(cp);
                            o.x += bscale * old.x;
                            o.y += bscale * old.y;
                            o.z += bscale * old.z;
                            o.w += bscale * old.w;
                        }
                        *reinterpret_cast<float4*>(cp) = o;
                    } else {
                        const float vv[4] = {v.x, v.y, v.z, v.w};
                        for (int j = 0; j < 4 && gcol + j < N; ++j) {
                            float o = alpha * vv[j];
                            if (bscale != 0.0f) o += bscale * cp[j];
                            cp[j] = o;
                        }
                    }
                }
                __syncwarp();
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(cluster_addr(smem_u32(&acc_empty[b]), 0));
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1 && rank == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (s_fail && lane == 0) {
            // Every MMA this pair issued must retire before the tensor memory is freed.
            umma_commit_pair(smem_u32(teardown));
            mbar_wait(smem_u32(teardown), 0);
        }
        __syncwarp();
    }
    // Neither CTA leaves (or frees its tensor memory) while the other may still
    // read its shared memory or write its tensor memory.
    cluster_sync_all();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P::kTmemCols) : "memory");
    }
}

template <int TN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
gemm_bf16x3_2sm_kernel(const __grid_constant__ GemmMaps maps, int M, int N, int KT, float alpha, float beta,
                       float* __restrict__ C, int64_t ldc, uint32_t* __restrict__ err) {
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the split pass launched before it
    gemm2_tile<TN>(maps, M, N, KT, alpha, beta, C, ldc, err, static_cast<int>(blockIdx.x >> 1));
}

// Grouped products: one launch over the tiles of up to kMaxGroup products of
// different shapes (the subtasks of a task, or the products of concurrent
// tasks).  Pair p takes tile p - tile_start[g] of product g, where g is the
// product whose range [tile_start[g], tile_start[g + 1]) holds p.
constexpr int kMaxGroup = 24;
struct Gemm2Product {
    GemmMaps maps;
    float* C;
    int64_t ldc;
    int M, N, KT;
    float alpha, beta;
};
struct Gemm2Group {
    Gemm2Product prod[kMaxGroup];
    int tile_start[kMaxGroup + 1];
    int count;
};
static_assert(sizeof(Gemm2Group) <= 32000, "kernel parameter space");

template <int TN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
gemm_bf16x3_2sm_grouped_kernel(const __grid_constant__ Gemm2Group grp, uint32_t* __restrict__ err) {
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the split passes launched before it
    const int pid = static_cast<int>(blockIdx.x >> 1);
    int g = 0;
    while (g + 1 < grp.count && pid >= grp.tile_start[g + 1]) ++g;
    const Gemm2Product& pr = grp.prod[g];
    gemm2_tile<TN>(pr.maps, pr.M, pr.N, pr.KT, pr.alpha, pr.beta, pr.C, pr.ldc, err, pid - grp.tile_start[g]);
}

// ---- 2-SM update kernel for short products (K <= 64) ------------------------
// With a single 64-deep K slice per tile (the LU trailing update, K = block
// size) the product is bound by reading and writing C, not by the MMAs.  The
// kernel above reads C with plain loads in its epilogue, a few in flight per
// thread, which leaves each SM far below its share of HBM bandwidth.  Here
// each epilogue warp issues TMA loads of its 32 rows of the C tile into shared
// memory at kernel start, so they overlap the operand loads and the MMAs,
// updates the tile in shared memory and writes each finished 32 x 32 box back
// with a TMA store (rows and columns outside M x N are neither read nor
// written).  Shared memory holds one operand stage (64 KB) and the CTA's
// 128 x 256 C tile (128 KB: 32 boxes of 32 x 32 fp32, SWIZZLE_128B, so that a
// warp's row-per-lane float4 accesses are free of bank conflicts).
constexpr int kBoxBytes = 32 * 32 * 4;
constexpr int kUpdCBytes = 128 * 256 * 4;
constexpr int kUpdSmemBytes = kStage2Bytes + kUpdCBytes + 1024 + 256;
constexpr uint32_t kUpdTmemCols = 256;

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
gemm_update_2sm_kernel(const __grid_constant__ GemmMaps maps, const __grid_constant__ CUtensorMap cmap, int M, int N,
                       float alpha, float beta, uint32_t* __restrict__ err) {
    // Launched as a programmatic dependent of the kernel that wrote the
    // operands (the split pass, or the LU panel solve), this returns once that
    // grid is complete and its writes are visible; otherwise it returns at once.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* ctile = smem + kStage2Bytes;  // 1024-byte aligned: kStage2Bytes is a multiple of 1024
    uint64_t* bars = reinterpret_cast<uint64_t*>(ctile + kUpdCBytes);
    uint64_t* full = bars;          // leader only: both CTAs' operand bytes
    uint64_t* acc_full = bars + 1;  // both CTAs: multicast commit after the MMAs
    uint64_t* cfull = bars + 2;     // [4] one per epilogue warp: its C rows landed
    uint64_t* teardown = bars + 6;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 7);
    __shared__ volatile int s_fail;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    int pm, pn;
    pair_tile(M, N, 256, static_cast<int>(blockIdx.x >> 1), pm, pn);
    const int m0 = pm * 256 + 128 * static_cast<int>(rank);
    const int n0 = pn * 256;
    const int nb0 = n0 + 128 * static_cast<int>(rank);

    if (threadIdx.x == 0) {
        s_fail = 0;
        mbar_init(smem_u32(full), 2);
        mbar_init(smem_u32(acc_full), 1);
        for (int q = 0; q < 4; ++q) mbar_init(smem_u32(&cfull[q]), 1);
        mbar_init(smem_u32(teardown), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kUpdTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    cluster_sync_all();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---- producer (both CTAs): the one K slice ----
        const uint32_t fbar = cluster_addr(smem_u32(full), 0);
        mbar_arrive_expect_tx_cluster(fbar, kStage2Bytes);
        tma_load_2d_pair(smem_u32(smem), &maps.ah, 0, m0, fbar);
        tma_load_2d_pair(smem_u32(smem + kHalf2), &maps.al, 0, m0, fbar);
        tma_load_2d_pair(smem_u32(smem + 2 * kHalf2), &maps.bh, 0, nb0, fbar);
        tma_load_2d_pair(smem_u32(smem + 3 * kHalf2), &maps.bl, 0, nb0, fbar);
    } else if (warp == 1 && lane == 0 && rank == 0) {
        // ---- MMA issuer (leader CTA) ----
        if (!mbar_wait(smem_u32(full), 0)) {
            s_fail = 1;
            atomicOr(err, kErrTimeout);
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = smem_u32(smem);
            const uint32_t a_hi = st, a_lo = st + kHalf2, b_hi = st + 2 * kHalf2, b_lo = st + 3 * kHalf2;
#pragma unroll
            for (int k16 = 0; k16 < BK2 / 16; ++k16) {
                const uint32_t off = k16 * 32;
                umma_bf16_pair_i(tmem, umma_desc_sw128(a_hi + off), umma_desc_sw128(b_hi + off), Pair2<256>::kIdesc, k16 != 0);
                umma_bf16_pair_i(tmem, umma_desc_sw128(a_hi + off), umma_desc_sw128(b_lo + off), Pair2<256>::kIdesc, 1u);
                umma_bf16_pair_i(tmem, umma_desc_sw128(a_lo + off), umma_desc_sw128(b_hi + off), Pair2<256>::kIdesc, 1u);
            }
            umma_commit_pair(smem_u32(acc_full));
        }
    } else if (warp >= 2) {
        // ---- epilogue (both CTAs): rows 32q .. 32q+31 of this CTA's 128 ----
        const int q = warp & 3;
        uint8_t* mine = ctile + q * 8 * kBoxBytes;
        const bool load_c = beta != 0.0f;
        const uint32_t cbar = smem_u32(&cfull[q]);
        if (lane == 0 && load_c) {
            mbar_expect_tx(cbar, 8 * kBoxBytes);
            for (int cb = 0; cb < 8; ++cb) tma_load_2d(smem_u32(mine + cb * kBoxBytes), &cmap, n0 + 32 * cb, m0 + 32 * q, cbar);
        }
        const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(acc_full), 0) && (!load_c || mbar_wait(cbar, 0)));
        if (!ok || s_fail) {
            s_fail = 1;
            atomicOr(err, kErrTimeout);
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int c = 0; c < 16; ++c) {
                uint32_t r[16];
                tmem_ld16(tmem + (static_cast<uint32_t>(32 * q) << 16) + 16 * c, r);
                const int cb = c >> 1, h = c & 1;
                uint8_t* rowp = mine + cb * kBoxBytes + lane * 128;  // this lane's row of the box
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float4* p = reinterpret_cast<float4*>(rowp + ((((h << 2) | j) ^ (lane & 7)) << 4));
                    float4 o = make_float4(alpha * __uint_as_float(r[4 * j]), alpha * __uint_as_float(r[4 * j + 1]),
                                           alpha * __uint_as_float(r[4 * j + 2]), alpha * __uint_as_float(r[4 * j + 3]));
                    if (load_c) {
                        const float4 old = *p;
                        o.x += beta * old.x;
                        o.y += beta * old.y;
                        o.z += beta * old.z;
                        o.w += beta * old.w;
                    }
                    *p = o;
                }
                if (h == 1) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) tma_store_2d(&cmap, n0 + 32 * cb, m0 + 32 * q, smem_u32(mine + cb * kBoxBytes));
                }
            }
            if (lane == 0) {
                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
            }
            __syncwarp();
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1 && rank == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (s_fail && lane == 0) {
            umma_commit_pair(smem_u32(teardown));
            mbar_wait(smem_u32(teardown), 0);
        }
        __syncwarp();
    }
    cluster_sync_all();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kUpdTmemCols) : "memory");
    }
}

// ---- split passes -----------------------------------------------------------
// Both splits in one launch: blocks [0, row_blocks) split the rows of A
// (M x K) as split_rows_kernel does, the others take one 32 x 32 tile of B
// (K x N) each as split_transpose_kernel does.  256 threads per block.
__global__ void __launch_bounds__(256)
split_both_kernel(const float* __restrict__ A, int64_t lda, int M, const float* __restrict__ B, int64_t ldb, int N,
                  int K, int Kp, int row_blocks, __nv_bfloat16* __restrict__ ah, __nv_bfloat16* __restrict__ al,
                  __nv_bfloat16* __restrict__ bh, __nv_bfloat16* __restrict__ bl) {
    // The product kernel is launched as a programmatic dependent of this pass:
    // let its launch begin (it waits for this grid before reading anything).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    __shared__ float t[32][33];
    if (static_cast<int>(blockIdx.x) < row_blocks) {
        const int64_t total = static_cast<int64_t>(M) * Kp;
        for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
             i += static_cast<int64_t>(row_blocks) * blockDim.x) {
            const int64_t r = i / Kp;
            const int k = static_cast<int>(i - r * Kp);
            const float x = k < K ? A[r * lda + k] : 0.0f;
            const __nv_bfloat16 h = __float2bfloat16_rn(x);
            ah[i] = h;
            al[i] = __float2bfloat16_rn(x - __bfloat162float(h));
        }
        return;
    }
    const int tile = blockIdx.x - row_blocks;
    const int tiles_n = (N + 31) / 32;
    const int k0 = (tile / tiles_n) * 32, n0 = (tile % tiles_n) * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int j = ty; j < 32; j += 8) {
        const int k = k0 + j, n = n0 + tx;
        t[j][tx] = (k < K && n < N) ? B[static_cast<int64_t>(k) * ldb + n] : 0.0f;
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int n = n0 + j, k = k0 + tx;
        if (n < N && k < Kp) {
            const float x = t[tx][j];
            const __nv_bfloat16 h = __float2bfloat16_rn(x);
            bh[static_cast<int64_t>(n) * Kp + k] = h;
            bl[static_cast<int64_t>(n) * Kp + k] = __float2bfloat16_rn(x - __bfloat162float(h));
        }
    }
}

__global__ void scale_kernel(float* C, int64_t ldc, int M, int N, float beta) {
    const int64_t total = static_cast<int64_t>(M) * N;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t r = i / N, c = i - r * N;
        float* p = C + r * ldc + c;
        *p = beta == 0.0f ? 0.0f : beta * *p;
    }
}

// ---- plain GPU form: FP32 SIMT GEMM, 64x64 tiles, 4x4 outputs per thread ------
__global__ void __launch_bounds__(256) sgemm_plain_kernel(int M, int N, int K, float alpha, const float* __restrict__ A,
                                                          int64_t lda, const float* __restrict__ B, int64_t ldb,
                                                          float beta, float* __restrict__ C, int64_t ldc) {
    __shared__ float As[16][64 + 1];
    __shared__ float Bs[16][64 + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int i = threadIdx.x; i < 16 * 64; i += 256) {
            const int kk = i / 64, mm = i % 64;
            As[kk][mm] = (m0 + mm < M && k0 + kk < K) ? A[static_cast<int64_t>(m0 + mm) * lda + k0 + kk] : 0.0f;
            Bs[kk][mm] = (n0 + mm < N && k0 + kk < K) ? B[static_cast<int64_t>(k0 + kk) * ldb + n0 + mm] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m < M && n < N) {
                float* p = C + static_cast<int64_t>(m) * ldc + n;
                *p = alpha * acc[i][j] + (beta != 0.0f ? beta * *p : 0.0f);
            }
        }
}

// ---- host side ----------------------------------------------------------------
using pmb::EncodeTiledFn;
EncodeTiledFn encode_fn() { return pmb::tensor_map_encoder(); }

// K-major bf16 operand [rows][kp]: boxes of box_k x box_rows, 64- or 128-byte swizzle.
int make_map(CUtensorMap* map, const void* base, int rows, int kp, int box_rows, int box_k = BK) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return pmb::fail(PMB_GRAPHICS_CARD_ERROR, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(kp), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(kp) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_k), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE,
                          box_k == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return pmb::fail(PMB_GRAPHICS_CARD_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return PMB_SUCCESS;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }
int padded_k(int K) { return (K + BK - 1) / BK * BK; }

// Launch on s as a programmatic dependent of the previous kernel when `dependent`.
template <typename... KArgs, typename... Args>
cudaError_t launch_dep(void (*kernel)(KArgs...), dim3 grid, int threads, int smem, cudaStream_t s, bool dependent,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = dependent ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Row-major fp32 C (M x N, ldc) in 32 x 32 boxes, SWIZZLE_128B; TMA needs a
// 16-byte aligned base and a row pitch that is a multiple of 16 bytes.
bool c_map_ok(const float* C, int64_t ldc) { return (reinterpret_cast<uintptr_t>(C) & 15) == 0 && (ldc & 3) == 0; }

int make_c_map(CUtensorMap* map, float* C, int M, int N, int64_t ldc) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return pmb::fail(PMB_GRAPHICS_CARD_ERROR, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(N), static_cast<cuuint64_t>(M)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ldc) * 4};
    const cuuint32_t box[2] = {32, 32};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return pmb::fail(PMB_GRAPHICS_CARD_ERROR, "cuTensorMapEncodeTiled (C) failed (%d)", (int)r);
    return PMB_SUCCESS;
}

// The short-product kernel on split operands ah/al (M x kp) and bh/bl (N x kp),
// kp <= 64, C satisfying c_map_ok.
int launch_update(int M, int N, int kp, float alpha, const __nv_bfloat16* ah, const __nv_bfloat16* al,
                  const __nv_bfloat16* bh, const __nv_bfloat16* bl, float beta, float* C, int64_t ldc, uint32_t* err,
                  cudaStream_t s, bool dependent = false) {
    GemmMaps maps;
    CUtensorMap cmap;
    int st;
    if ((st = make_map(&maps.ah, ah, M, kp, 128, BK2)) != PMB_SUCCESS) return st;
    if ((st = make_map(&maps.al, al, M, kp, 128, BK2)) != PMB_SUCCESS) return st;
    if ((st = make_map(&maps.bh, bh, N, kp, 128, BK2)) != PMB_SUCCESS) return st;
    if ((st = make_map(&maps.bl, bl, N, kp, 128, BK2)) != PMB_SUCCESS) return st;
    if ((st = make_c_map(&cmap, C, M, N, ldc)) != PMB_SUCCESS) return st;
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(gemm_update_2sm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kUpdSmemBytes);
        if (attr_err == cudaSuccess &&
            pmb::tmem_exclusive(reinterpret_cast<const void*>(gemm_update_2sm_kernel), kThreads, kUpdSmemBytes,
                                "gemm_update_2sm_kernel") != PMB_SUCCESS)
            attr_err = cudaErrorInvalidConfiguration;
    });
    PMB_CUDA_TRY(attr_err);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * ((M + 255) / 256) * ((N + 255) / 256));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kUpdSmemBytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = dependent ? 1 : 0;
    PMB_CUDA_TRY(cudaLaunchKernelEx(&cfg, gemm_update_2sm_kernel, maps, cmap, M, N, alpha, beta, err));
    return PMB_SUCCESS;
}

}  // namespace

extern "C" size_t pmb_gemm_workspace_bytes(int M, int N, int K) {
    if (M <= 0 || N <= 0 || K <= 0) return 256;
    const size_t kp = padded_k(K);
    return 256 + 2 * align256(static_cast<size_t>(M) * kp * 2) + 2 * align256(static_cast<size_t>(N) * kp * 2);
}

namespace pmb {

// The GEMM behind pmb_sgemm_bf16x3.  A and B are copied into the split buffers
// of the workspace before the product runs, so C may overlap A or B (the LU
// panel solves write their result over their own operand).  clear_error=false
// skips clearing the workspace's error word (a caller issuing many products on
// one workspace clears it once).
int sgemm_bf16x3_launch(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                        float beta, float* C, int64_t ldc, void* workspace, size_t ws_bytes, cudaStream_t s,
                        bool clear_error);

// C = alpha * (Ahi + Alo)(Bhi + Blo)^T + beta * C without the split pass, for a
// caller that already holds the split operands: ah/al M x kp and bh/bl N x kp,
// K-major bf16 with zero padding beyond K, kp a multiple of 8 and at most 64.
// C (row-major, ldc) must have a 16-byte aligned base and ldc a multiple of 4.
// Errors of the kernel are OR-ed into *err.  dependent = launch as a
// programmatic dependent of the previous kernel on s: the kernel waits for
// that grid to complete before it touches any data, so only the launch
// latency overlaps the previous kernel.
int gemm_presplit_launch(int M, int N, int kp, float alpha, const __nv_bfloat16* ah, const __nv_bfloat16* al,
                         const __nv_bfloat16* bh, const __nv_bfloat16* bl, float beta, float* C, int64_t ldc,
                         uint32_t* err, cudaStream_t s, bool dependent);

}  // namespace pmb

int pmb::gemm_presplit_launch(int M, int N, int kp, float alpha, const __nv_bfloat16* ah, const __nv_bfloat16* al,
                              const __nv_bfloat16* bh, const __nv_bfloat16* bl, float beta, float* C, int64_t ldc,
                              uint32_t* err, cudaStream_t s, bool dependent) {
    PMB_CHECK_ARG(M >= 0 && N >= 0, "negative GEMM size");
    if (M == 0 || N == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(kp > 0 && kp <= BK2 && kp % 8 == 0, "split depth %d: need a multiple of 8 up to %d", kp, BK2);
    PMB_CHECK_ARG(ah && al && bh && bl && C && err, "null pointer");
    PMB_CHECK_ARG(ldc >= N && c_map_ok(C, ldc), "C needs a 16-byte aligned base and ldc a multiple of 4");
    return launch_update(M, N, kp, alpha, ah, al, bh, bl, beta, C, ldc, err, s, dependent);
}

extern "C" int pmb_sgemm_bf16x3(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B,
                                int64_t ldb, float beta, float* C, int64_t ldc, void* workspace, size_t ws_bytes,
                                void* stream) {
    return pmb::sgemm_bf16x3_launch(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, workspace, ws_bytes,
                                    static_cast<cudaStream_t>(stream), true);
}

namespace {

// Product kernels of the BF16x3 GEMM: 128 x 256 tiles per CTA, or 256 x 256 /
// 256 x 128 tiles per CTA pair.
enum class GemmCfg : int { kOneSm = 0, kPair256 = 1, kPair128 = 2 };

int launch_product(GemmCfg cfg, int M, int N, int kp, float alpha, const __nv_bfloat16* ah, const __nv_bfloat16* al,
                   const __nv_bfloat16* bh, const __nv_bfloat16* bl, float beta, float* C, int64_t ldc, uint32_t* err,
                   cudaStream_t s) {
    GemmMaps maps;
    int st;
    if (cfg != GemmCfg::kOneSm) {
        const int tn = cfg == GemmCfg::kPair128 ? 128 : 256;
        if ((st = make_map(&maps.ah, ah, M, kp, 128, BK2)) != PMB_SUCCESS) return st;
        if ((st = make_map(&maps.al, al, M, kp, 128, BK2)) != PMB_SUCCESS) return st;
        if ((st = make_map(&maps.bh, bh, N, kp, tn / 2, BK2)) != PMB_SUCCESS) return st;
        if ((st = make_map(&maps.bl, bl, N, kp, tn / 2, BK2)) != PMB_SUCCESS) return st;
        static std::once_flag attr2_once;
        static cudaError_t attr2_err = cudaSuccess;
        std::call_once(attr2_once, [] {
            attr2_err = cudaFuncSetAttribute(gemm_bf16x3_2sm_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             Pair2<256>::kSmemBytes);
            if (attr2_err == cudaSuccess)
                attr2_err = cudaFuncSetAttribute(gemm_bf16x3_2sm_kernel<128>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, Pair2<128>::kSmemBytes);
            if (attr2_err == cudaSuccess &&
                (pmb::tmem_exclusive(reinterpret_cast<const void*>(gemm_bf16x3_2sm_kernel<256>), kThreads,
                                     Pair2<256>::kSmemBytes, "gemm_bf16x3_2sm_kernel<256>") != PMB_SUCCESS ||
                 pmb::tmem_exclusive(reinterpret_cast<const void*>(gemm_bf16x3_2sm_kernel<128>), kThreads,
                                     Pair2<128>::kSmemBytes, "gemm_bf16x3_2sm_kernel<128>") != PMB_SUCCESS))
                attr2_err = cudaErrorInvalidConfiguration;
        });
        PMB_CUDA_TRY(attr2_err);
        const dim3 grid2(2 * ((M + 255) / 256) * ((N + tn - 1) / tn));
        if (tn == 128)
            PMB_CUDA_TRY(launch_dep(gemm_bf16x3_2sm_kernel<128>, grid2, kThreads, Pair2<128>::kSmemBytes, s, true, maps,
                                    M, N, (kp + BK2 - 1) / BK2, alpha, beta, C, ldc, err));
        else
            PMB_CUDA_TRY(launch_dep(gemm_bf16x3_2sm_kernel<256>, grid2, kThreads, Pair2<256>::kSmemBytes, s, true, maps,
                                    M, N, (kp + BK2 - 1) / BK2, alpha, beta, C, ldc, err));
        return PMB_SUCCESS;
    }
    if ((st = make_map(&maps.ah, ah, M, kp, BM)) != PMB_SUCCESS) return st;
    if ((st = make_map(&maps.al, al, M, kp, BM)) != PMB_SUCCESS) return st;
    if ((st = make_map(&maps.bh, bh, N, kp, BN)) != PMB_SUCCESS) return st;
    if ((st = make_map(&maps.bl, bl, N, kp, BN)) != PMB_SUCCESS) return st;
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(gemm_bf16x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (attr_err == cudaSuccess &&
            pmb::tmem_exclusive(reinterpret_cast<const void*>(gemm_bf16x3_kernel), kThreads, kSmemBytes,
                                "gemm_bf16x3_kernel") != PMB_SUCCESS)
            attr_err = cudaErrorInvalidConfiguration;
    });
    PMB_CUDA_TRY(attr_err);
    const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    PMB_CUDA_TRY(launch_dep(gemm_bf16x3_kernel, grid, kThreads, kSmemBytes, s, true, maps, M, N, kp / BK, alpha, beta, C,
                            ldc, err));
    return PMB_SUCCESS;
}

int sm_pair_count() {
    static const int pairs = [] {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            sms = 148;
        }
        return sms / 2;
    }();
    return pairs;
}

// The fixed rule: CTA pairs for M > 128, with 256 x 128 tiles when 256 x 256
// ones would leave at least half the SM pairs without a tile (e.g. 1024 x
// 1024: 16 tiles for 74 pairs); one CTA per 128 x 256 tile otherwise.
GemmCfg rule_cfg(int M, int N) {
    if (M <= BM) return GemmCfg::kOneSm;
    const int64_t tiles256 = static_cast<int64_t>((M + 255) / 256) * ((N + 255) / 256);
    return 2 * tiles256 <= sm_pair_count() ? GemmCfg::kPair128 : GemmCfg::kPair256;
}

int ceil_log2(int64_t x) {
    int l = 0;
    while ((int64_t{1} << l) < x) ++l;
    return l;
}

// Autotuner (PMB_GEMM_AUTOTUNE=1): the first product of each shape class
// (ceil log2 of M, N and the padded K) times the three product kernels on the
// call's own operands -- only when C is write-only (beta = 0) and the stream
// is not being captured -- and remembers the fastest; later products of the
// class use it.  Each timed kernel writes all of C, so the call's result is
// the last one's.  Off (the default), or for a class not tuned, the fixed rule.
GemmCfg choose_cfg(int M, int N, int kp, float alpha, const __nv_bfloat16* ah, const __nv_bfloat16* al,
                   const __nv_bfloat16* bh, const __nv_bfloat16* bl, float beta, float* C, int64_t ldc, uint32_t* err,
                   cudaStream_t s) {
    static const bool tune = [] {
        const char* v = getenv("PMB_GEMM_AUTOTUNE");
        return v && v[0] == '1';
    }();
    const GemmCfg rule = rule_cfg(M, N);
    if (!tune) return rule;
    const uint32_t key = (static_cast<uint32_t>(ceil_log2(M)) << 16) | (static_cast<uint32_t>(ceil_log2(N)) << 8) |
                         static_cast<uint32_t>(ceil_log2(kp));
    static std::mutex mu;
    static std::map<uint32_t, GemmCfg> best;
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = best.find(key);
        if (it != best.end()) return it->second;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (beta != 0.0f || cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return rule;
    }
    const GemmCfg cand[3] = {GemmCfg::kOneSm, GemmCfg::kPair256, GemmCfg::kPair128};
    cudaEvent_t ev[4] = {};
    for (cudaEvent_t& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            for (cudaEvent_t& x : ev)
                if (x) cudaEventDestroy(x);
            return rule;
        }
    bool ok = launch_product(rule, M, N, kp, alpha, ah, al, bh, bl, beta, C, ldc, err, s) == PMB_SUCCESS;  // warm-up
    ok = ok && cudaEventRecord(ev[0], s) == cudaSuccess;
    for (int i = 0; i < 3 && ok; ++i) {
        ok = launch_product(cand[i], M, N, kp, alpha, ah, al, bh, bl, beta, C, ldc, err, s) == PMB_SUCCESS;
        ok = ok && cudaEventRecord(ev[i + 1], s) == cudaSuccess;
    }
    GemmCfg pick = rule;
    if (ok && cudaEventSynchronize(ev[3]) == cudaSuccess) {
        float best_ms = 0.0f;
        for (int i = 0; i < 3; ++i) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) != cudaSuccess) continue;
            if (i == 0 || ms < best_ms) {
                best_ms = ms;
                pick = cand[i];
            }
        }
        std::lock_guard<std::mutex> g(mu);
        best[key] = pick;
    }
    cudaGetLastError();
    for (cudaEvent_t& e : ev) cudaEventDestroy(e);
    return pick;
}

}  // namespace

int pmb::sgemm_bf16x3_launch(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B,
                             int64_t ldb, float beta, float* C, int64_t ldc, void* workspace, size_t ws_bytes,
                             cudaStream_t s, bool clear_error) {
    PMB_CHECK_ARG(M >= 0 && N >= 0 && K >= 0, "negative GEMM size");
    if (M == 0 || N == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(C && workspace && (K == 0 || (A && B)), "null pointer");
    PMB_CHECK_ARG(ldc >= N && (K == 0 || (lda >= K && ldb >= N)), "leading dimension too small");
    PMB_CHECK_ARG((reinterpret_cast<uintptr_t>(workspace) & 255) == 0, "workspace must be 256-byte aligned");
    PMB_CHECK_ARG(ws_bytes >= pmb_gemm_workspace_bytes(M, N, K), "GEMM workspace %zu bytes, need %zu", ws_bytes,
                  pmb_gemm_workspace_bytes(M, N, K));
    if (K == 0) {
        scale_kernel<<<256, 256, 0, s>>>(C, ldc, M, N, beta);
        PMB_CUDA_TRY(cudaGetLastError());
        return PMB_SUCCESS;
    }
    const int kp = padded_k(K);
    char* ws = static_cast<char*>(workspace);
    uint32_t* err = reinterpret_cast<uint32_t*>(ws) + 1;
    __nv_bfloat16* ah = reinterpret_cast<__nv_bfloat16*>(ws + 256);
    __nv_bfloat16* al = reinterpret_cast<__nv_bfloat16*>(ws + 256 + align256(static_cast<size_t>(M) * kp * 2));
    __nv_bfloat16* bh = reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(al) + align256(static_cast<size_t>(M) * kp * 2));
    __nv_bfloat16* bl = reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(bh) + align256(static_cast<size_t>(N) * kp * 2));

    if (clear_error) PMB_CUDA_TRY(cudaMemsetAsync(ws, 0, 256, s));
    {
        const int64_t row_elems = static_cast<int64_t>(M) * kp;
        const int row_blocks = static_cast<int>(std::min<int64_t>(1184, (row_elems + 255) / 256));
        const int tiles = ((N + 31) / 32) * ((kp + 31) / 32);
        split_both_kernel<<<row_blocks + tiles, 256, 0, s>>>(A, lda, M, B, ldb, N, K, kp, row_blocks, ah, al, bh, bl);
        PMB_CUDA_TRY(cudaGetLastError());
    }

    // PMB_GEMM_KERNEL=1sm keeps the 1-SM kernel for every shape.
    static const bool force_1sm = [] {
        const char* v = getenv("PMB_GEMM_KERNEL");
        return v && std::string(v) == "1sm";
    }();
    // A single K slice: bound by C traffic, read and written by TMA.
    if (kp <= BK2 && c_map_ok(C, ldc) && !force_1sm)
        return launch_update(M, N, kp, alpha, ah, al, bh, bl, beta, C, ldc, err, s, true);

    if (force_1sm) return launch_product(GemmCfg::kOneSm, M, N, kp, alpha, ah, al, bh, bl, beta, C, ldc, err, s);
    return launch_product(choose_cfg(M, N, kp, alpha, ah, al, bh, bl, beta, C, ldc, err, s), M, N, kp, alpha, ah, al,
                          bh, bl, beta, C, ldc, err, s);
}

extern "C" int pmb_sgemm_plain(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B,
                               int64_t ldb, float beta, float* C, int64_t ldc, void* stream) {
    PMB_CHECK_ARG(M >= 0 && N >= 0 && K >= 0, "negative GEMM size");
    if (M == 0 || N == 0) return PMB_SUCCESS;
    PMB_CHECK_ARG(C && (K == 0 || (A && B)), "null pointer");
    sgemm_plain_kernel<<<dim3((N + 63) / 64, (M + 63) / 64), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

// ---------------------------------------------------------------------------
// Grouped products: many C = alpha A B + beta C of different shapes in one
// launch of the product kernel (after one split pass per product), instead of
// a split + product launch pair per product.

namespace {

size_t grouped_ws_bytes(const pmb_gemm_problem* probs, int count) {
    size_t total = 256;
    for (int i = 0; i < count; ++i) {
        const pmb_gemm_problem& q = probs[i];
        if (q.M <= 0 || q.N <= 0 || q.K <= 0) continue;
        total += pmb_gemm_workspace_bytes(q.M, q.N, q.K) - 256;
    }
    return total;
}

}  // namespace

extern "C" size_t pmb_gemm_grouped_workspace_bytes(const pmb_gemm_problem* problems, int count) {
    if (!problems || count <= 0) return 256;
    return grouped_ws_bytes(problems, count);
}

extern "C" int pmb_sgemm_bf16x3_grouped(const pmb_gemm_problem* problems, int count, void* workspace,
                                        size_t workspace_bytes, void* stream) {
    PMB_CHECK_ARG(problems && count >= 0, "null problem list");
    PMB_CHECK_ARG(workspace && (reinterpret_cast<uintptr_t>(workspace) & 255) == 0,
                  "workspace must be non-null and 256-byte aligned");
    PMB_CHECK_ARG(workspace_bytes >= grouped_ws_bytes(problems, count), "grouped GEMM workspace %zu bytes, need %zu",
                  workspace_bytes, grouped_ws_bytes(problems, count));
    for (int i = 0; i < count; ++i) {
        const pmb_gemm_problem& q = problems[i];
        PMB_CHECK_ARG(q.M >= 0 && q.N >= 0 && q.K >= 0, "problem %d: negative size", i);
        if (q.M == 0 || q.N == 0) continue;
        PMB_CHECK_ARG(q.C && (q.K == 0 || (q.A && q.B)), "problem %d: null pointer", i);
        PMB_CHECK_ARG(q.ldc >= q.N && (q.K == 0 || (q.lda >= q.K && q.ldb >= q.N)),
                      "problem %d: leading dimension too small", i);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(workspace);
    uint32_t* err = reinterpret_cast<uint32_t*>(ws) + 1;
    PMB_CUDA_TRY(cudaMemsetAsync(ws, 0, 256, s));
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(gemm_bf16x3_2sm_grouped_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        Pair2<256>::kSmemBytes);
        if (attr_err == cudaSuccess)
            attr_err = cudaFuncSetAttribute(gemm_bf16x3_2sm_grouped_kernel<128>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, Pair2<128>::kSmemBytes);
        if (attr_err == cudaSuccess &&
            (pmb::tmem_exclusive(reinterpret_cast<const void*>(gemm_bf16x3_2sm_grouped_kernel<256>), kThreads,
                                 Pair2<256>::kSmemBytes, "gemm_bf16x3_2sm_grouped_kernel<256>") != PMB_SUCCESS ||
             pmb::tmem_exclusive(reinterpret_cast<const void*>(gemm_bf16x3_2sm_grouped_kernel<128>), kThreads,
                                 Pair2<128>::kSmemBytes, "gemm_bf16x3_2sm_grouped_kernel<128>") != PMB_SUCCESS))
            attr_err = cudaErrorInvalidConfiguration;
    });
    PMB_CUDA_TRY(attr_err);
    static const int sm_pairs = [] {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            sms = 148;
        }
        return sms / 2;
    }();

    // Split every product into its bf16 hi/lo operands (workspace laid out in
    // problem order); K == 0 products only scale C.
    struct Split {
        const __nv_bfloat16 *ah, *al, *bh, *bl;
        int kp;
    };
    std::vector<Split> split(static_cast<size_t>(count));
    std::vector<int> live;
    size_t off = 256;
    for (int i = 0; i < count; ++i) {
        const pmb_gemm_problem& q = problems[i];
        if (q.M == 0 || q.N == 0) continue;
        if (q.K == 0) {
            scale_kernel<<<256, 256, 0, s>>>(q.C, q.ldc, q.M, q.N, q.beta);
            PMB_CUDA_TRY(cudaGetLastError());
            continue;
        }
        const int kp = padded_k(q.K);
        const size_t a_bytes = align256(static_cast<size_t>(q.M) * kp * 2);
        const size_t b_bytes = align256(static_cast<size_t>(q.N) * kp * 2);
        __nv_bfloat16* ah = reinterpret_cast<__nv_bfloat16*>(ws + off);
        __nv_bfloat16* al = reinterpret_cast<__nv_bfloat16*>(ws + off + a_bytes);
        __nv_bfloat16* bh = reinterpret_cast<__nv_bfloat16*>(ws + off + 2 * a_bytes);
        __nv_bfloat16* bl = reinterpret_cast<__nv_bfloat16*>(ws + off + 2 * a_bytes + b_bytes);
        off += 2 * a_bytes + 2 * b_bytes;
        const int64_t row_elems = static_cast<int64_t>(q.M) * kp;
        const int row_blocks = static_cast<int>(std::min<int64_t>(1184, (row_elems + 255) / 256));
        const int tiles = ((q.N + 31) / 32) * ((kp + 31) / 32);
        split_both_kernel<<<row_blocks + tiles, 256, 0, s>>>(q.A, q.lda, q.M, q.B, q.ldb, q.N, q.K, kp, row_blocks, ah,
                                                             al, bh, bl);
        PMB_CUDA_TRY(cudaGetLastError());
        split[i] = Split{ah, al, bh, bl, kp};
        live.push_back(i);
    }
    // The products, kMaxGroup per launch, each launch a programmatic
    // dependent of the work before it on the stream.
    for (size_t g0 = 0; g0 < live.size(); g0 += kMaxGroup) {
        const size_t g1 = std::min(live.size(), g0 + kMaxGroup);
        int64_t tiles256 = 0;
        for (size_t j = g0; j < g1; ++j) {
            const pmb_gemm_problem& q = problems[live[j]];
            tiles256 += static_cast<int64_t>((q.M + 255) / 256) * ((q.N + 255) / 256);
        }
        // 256 x 128 tiles when 256 x 256 ones would leave at least half the SM pairs idle.
        const bool narrow = 2 * tiles256 <= sm_pairs;
        const int tn = narrow ? 128 : 256;
        Gemm2Group grp;
        grp.count = static_cast<int>(g1 - g0);
        int total = 0, st;
        for (int j = 0; j < grp.count; ++j) {
            const pmb_gemm_problem& q = problems[live[g0 + j]];
            const Split& sp = split[live[g0 + j]];
            Gemm2Product& pr = grp.prod[j];
            if ((st = make_map(&pr.maps.ah, sp.ah, q.M, sp.kp, 128, BK2)) != PMB_SUCCESS) return st;
            if ((st = make_map(&pr.maps.al, sp.al, q.M, sp.kp, 128, BK2)) != PMB_SUCCESS) return st;
            if ((st = make_map(&pr.maps.bh, sp.bh, q.N, sp.kp, tn / 2, BK2)) != PMB_SUCCESS) return st;
            if ((st = make_map(&pr.maps.bl, sp.bl, q.N, sp.kp, tn / 2, BK2)) != PMB_SUCCESS) return st;
            pr.C = q.C;
            pr.ldc = q.ldc;
            pr.M = q.M;
            pr.N = q.N;
            pr.KT = (sp.kp + BK2 - 1) / BK2;
            pr.alpha = q.alpha;
            pr.beta = q.beta;
            grp.tile_start[j] = total;
            total += ((q.M + 255) / 256) * ((q.N + tn - 1) / tn);
        }
        grp.tile_start[grp.count] = total;
        if (narrow)
            PMB_CUDA_TRY(launch_dep(gemm_bf16x3_2sm_grouped_kernel<128>, dim3(2 * total), kThreads,
                                    Pair2<128>::kSmemBytes, s, true, grp, err));
        else
            PMB_CUDA_TRY(launch_dep(gemm_bf16x3_2sm_grouped_kernel<256>, dim3(2 * total), kThreads,
                                    Pair2<256>::kSmemBytes, s, true, grp, err));
    }
    return PMB_SUCCESS;
}
