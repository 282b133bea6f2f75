// imageFiltering subtask kernel for sm_100a.
//
// Computes, for every output pixel (i, j) of a subtask rectangle and every
// channel c, the (2R+1)^2 stencil of testSuite/imageFiltering/source/code/src/
// imageFiltering.cpp:419-468 (imageFilter_cpu):
//
//     out[i][j][c] = sum_{ky,kx} img[clamp(i+ky-R)][clamp(j+kx-R)][2-c] * f[ky][kx]
//
// where img[m][n][ch] is byte ch of pixel n in buffer row H-1-m (the address
// space stores the image bottom-up, :438) and clamp() is edge replication
// (:433-434).  WRAP mode keeps the reference's signed-char accumulator (the
// byte is the sum mod 256); CLAMP mode sums unsigned bytes exactly and clamps
// to [0, 255].
//
// Two kernels: imgf_tc_kernel (tensor cores, below) for R <= 8 -- every
// radius the reference's own runs use -- and imgf_kernel, the generic dp4a
// form, for 9 <= R <= 15.  The batch of subtasks (items) of one or several
// tasks runs in ONE launch.
//
// Generic form.  One CTA owns a 64 x 32 output tile.  It stages the tile
// plus halo once into shared memory as three planar byte planes (one per
// output channel), de-interleaving RGB with byte permutes.  Each thread then
// produces a 4-pixel x 4-row block: for every staged row it reads a few
// aligned 32-bit words of a plane and feeds them to dp4a (4 byte
// multiply-adds per instruction) against filter "pattern" words precomputed
// on the host (filter row ky shifted so that tap kx lines up with the byte it
// multiplies).  blockIdx.x is mapped to (item, tile).
#include <algorithm>
#include <mutex>

#include "pmb_common.cuh"

namespace {

constexpr int kTW = 64;                    // tile width (pixels)
constexpr int kTH = 32;                    // tile height (rows)
constexpr int kV = 4;                      // output rows per thread
constexpr int kGX = kTW / 4;               // 4-pixel groups per tile row
constexpr int kThreads = kGX * (kTH / kV); // 128

template <int R>
struct Geo {
    static constexpr int KD = 2 * R + 1;             // filter taps per row
    static constexpr int PADL = ((R + 3) / 4) * 4;   // left halo, word aligned
    static constexpr int OFF = PADL - R;             // first tap byte of pixel 0 in its window
    static constexpr int NW = (OFF + 2 * R + 3) / 4 + 1;  // 32-bit words in a 4-pixel window
    static constexpr int PW = kTW + PADL + 4 * NW;   // plane row width (bytes)
    static constexpr int PH = kTH + 2 * R;           // plane rows
    static constexpr int GPR = PW / 4;               // 4-pixel groups per plane row
};

// Does output pixel k (0..3) of a group have taps inside window word w?
template <int R>
__host__ __device__ constexpr bool tap_word_used(int k, int w) {
    return 4 * w <= Geo<R>::OFF + k + 2 * R && 4 * w + 3 >= Geo<R>::OFF + k;
}

template <int R, int MAXI>
struct ImgfParams {
    uint32_t pat[Geo<R>::KD][4][Geo<R>::NW];
    int n_items;
    int tile_start[MAXI + 1];
    int tiles_x[MAXI];
    pmb_imgf_item items[MAXI];
};

__device__ __forceinline__ int dp4a_us(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

template <int R, int MODE, int MAXI>
__global__ void __launch_bounds__(kThreads)
imgf_kernel(const __grid_constant__ ImgfParams<R, MAXI> p) {
    using G = Geo<R>;
    __shared__ __align__(16) uint8_t planes[3][G::PH][G::PW];

    // ---- which item / tile ------------------------------------------------
    const int t = blockIdx.x;
    int lo = 0, hi = p.n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.tile_start[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const pmb_imgf_item& it = p.items[lo];
    const int local = t - p.tile_start[lo];
    const int tx = local % p.tiles_x[lo];
    const int ty = local / p.tiles_x[lo];
    const int tile_c0 = it.c0 + tx * kTW;
    const int tile_r0 = it.r0 + ty * kTH;
    const int H = it.height;
    const int mlo = max(0, it.r0 - R), mhi = min(H - 1, it.r1 - 1 + R);
    const int clo = max(0, it.c0 - R), chi = min(it.width - 1, it.c1 - 1 + R);

    // ---- stage tile + halo as planes: plane c holds input byte 2-c ---------
    const uint8_t* inb = it.in;
    const int64_t ip = it.in_pitch;
    const bool al4 = ((reinterpret_cast<uintptr_t>(inb) | static_cast<uintptr_t>(ip)) & 3) == 0;
    for (int g = threadIdx.x; g < G::PH * G::GPR; g += kThreads) {
        const int yy = g / G::GPR;
        const int xg = g - yy * G::GPR;
        const int m = pmb::clampi(tile_r0 - R + yy, mlo, mhi);
        const uint8_t* rowp = inb + static_cast<int64_t>(H - 1 - m - it.in_row0) * ip;
        const int n0 = tile_c0 - G::PADL + 4 * xg;
        uint32_t o0, o1, o2;
        if (al4 && n0 >= clo && n0 + 3 <= chi && ((n0 - it.in_col0) & 3) == 0) {
            const uint32_t* s = reinterpret_cast<const uint32_t*>(rowp + 3 * (n0 - it.in_col0));
            const uint32_t w0 = __ldg(s), w1 = __ldg(s + 1), w2 = __ldg(s + 2);
            // Pixel q's bytes b0 b1 b2 sit at 3q..3q+2 of the 12-byte quad.
            o0 = __byte_perm(__byte_perm(w0, w1, 0x0052), w2, 0x7410);  // b2 of pixels 0..3
            o1 = __byte_perm(__byte_perm(w0, w1, 0x0741), w2, 0x6210);  // b1
            o2 = __byte_perm(__byte_perm(w0, w1, 0x0630), w2, 0x5210);  // b0
        } else {
            o0 = o1 = o2 = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int n = pmb::clampi(n0 + q, clo, chi);
                const uint8_t* px = rowp + 3 * (n - it.in_col0);
                o0 |= static_cast<uint32_t>(__ldg(px + 2)) << (8 * q);
                o1 |= static_cast<uint32_t>(__ldg(px + 1)) << (8 * q);
                o2 |= static_cast<uint32_t>(__ldg(px + 0)) << (8 * q);
            }
        }
        *reinterpret_cast<uint32_t*>(&planes[0][yy][4 * xg]) = o0;
        *reinterpret_cast<uint32_t*>(&planes[1][yy][4 * xg]) = o1;
        *reinterpret_cast<uint32_t*>(&planes[2][yy][4 * xg]) = o2;
    }
    __syncthreads();

    // ---- 4 pixels x kV rows per thread, dp4a over plane words -------------
    const int gx = threadIdx.x % kGX;
    const int gy = threadIdx.x / kGX;
    uint32_t res[kV][4];
#pragma unroll
    for (int v = 0; v < kV; ++v)
#pragma unroll
        for (int k = 0; k < 4; ++k) res[v][k] = 0;

#pragma unroll 1
    for (int ch = 0; ch < 3; ++ch) {
        int acc[kV][4];
#pragma unroll
        for (int v = 0; v < kV; ++v)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[v][k] = 0;

#pragma unroll 1
        for (int yy = 0; yy < kV + 2 * R; ++yy) {
            const uint32_t* rp =
                reinterpret_cast<const uint32_t*>(&planes[ch][gy * kV + yy][4 * gx]);
            uint32_t win[G::NW];
#pragma unroll
            for (int w = 0; w < G::NW; ++w) win[w] = rp[w];
#pragma unroll
            for (int v = 0; v < kV; ++v) {
                const int ky = yy - v;
                if (ky < 0 || ky >= G::KD) continue;
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int w = 0; w < G::NW; ++w)
                        if (tap_word_used<R>(k, w))
                            acc[v][k] = dp4a_us(win[w], p.pat[ky][k][w], acc[v][k]);
            }
        }

#pragma unroll
        for (int v = 0; v < kV; ++v)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int a = acc[v][k];
                const uint32_t b = MODE == PMB_IMGF_WRAP ? static_cast<uint32_t>(a) & 0xffu
                                                         : static_cast<uint32_t>(min(max(a, 0), 255));
                res[v][k] |= b << (8 * ch);
            }
    }

    // ---- write: pixel k's channels (c0 c1 c2) are bytes 3k..3k+2 -----------
    const int j0 = tile_c0 + 4 * gx;
    if (j0 >= it.c1) return;
#pragma unroll
    for (int v = 0; v < kV; ++v) {
        const int i = tile_r0 + gy * kV + v;
        if (i >= it.r1) break;
        uint8_t* dst = it.out + static_cast<int64_t>(i - it.out_row0) * it.out_pitch +
                       3 * (j0 - it.out_col0);
        if (j0 + 3 < it.c1 && (reinterpret_cast<uintptr_t>(dst) & 3) == 0) {
            uint32_t* d = reinterpret_cast<uint32_t*>(dst);
            d[0] = res[v][0] | (res[v][1] << 24);
            d[1] = (res[v][1] >> 8) | (res[v][2] << 16);
            d[2] = (res[v][2] >> 16) | (res[v][3] << 8);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (j0 + k >= it.c1) break;
                dst[3 * k + 0] = static_cast<uint8_t>(res[v][k]);
                dst[3 * k + 1] = static_cast<uint8_t>(res[v][k] >> 8);
                dst[3 * k + 2] = static_cast<uint8_t>(res[v][k] >> 16);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Byte packing shared by the tensor-core path.

// Four 32-bit sums into four bytes (sum k -> byte k): CLAMP saturates to
// [0, 255] with cvt.pack.sat (two sums per instruction), WRAP keeps the low
// byte of each sum.
template <int MODE>
__device__ __forceinline__ uint32_t pack4(const int (&a)[4]) {
    if (MODE == PMB_IMGF_CLAMP) {
        uint32_t hi, d;
        asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, %3;" : "=r"(hi) : "r"(a[3]), "r"(a[2]), "r"(0));
        asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a[1]), "r"(a[0]), "r"(hi));
        return d;
    }
    const uint32_t lo = __byte_perm(static_cast<uint32_t>(a[0]), static_cast<uint32_t>(a[1]), 0x0040);
    const uint32_t hi = __byte_perm(static_cast<uint32_t>(a[2]), static_cast<uint32_t>(a[3]), 0x0040);
    return __byte_perm(lo, hi, 0x5410);
}

// De-interleave a 12-byte RGB quad (pixels q0..q3) into the three plane words
// (plane c holds input byte 2-c).
__device__ __forceinline__ void deinterleave4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t& o0, uint32_t& o1,
                                              uint32_t& o2) {
    o0 = __byte_perm(__byte_perm(w0, w1, 0x0052), w2, 0x7410);
    o1 = __byte_perm(__byte_perm(w0, w1, 0x0741), w2, 0x6210);
    o2 = __byte_perm(__byte_perm(w0, w1, 0x0630), w2, 0x5210);
}

// ---------------------------------------------------------------------------
// Tensor-core path for R <= 8: the stencil as int8 matrix products on the
// 5th-generation tensor cores (tcgen05.mma kind::i8, u8 pixels x s8 weights,
// exact s32 sums in tensor memory), so integer parity is unchanged.
//
// Output tiles are TH rows x 64 pixels.  Per channel plane P and filter
// row ky a tile is D += A_ky * B_ky with
//   A_ky[i][k] = P[i + ky][16t - 8 + k]            (M = 128 rows, K = 32 columns)
//   B_ky[k][j] = f[ky][k - j + R - 8]  (zero outside [0, 2R])     (N = 16 output columns)
// for each 16-column group t: the 32-column window of input bytes times a
// banded Toeplitz slice of the filter row (plane row r = image row
// tile_r0 - R + r, plane column x = pixel tile_c0 + x).  An MMA whose A
// comes from shared memory costs as long as reading its 4 KB there, so A
// lives in tensor memory instead: the staging threads de-interleave each
// input row in registers and write it straight into TMEM (tcgen05.st, one
// lane per thread: five 16-column chunks = 20 columns per channel), and the
// ky shift is applied there with tcgen05.shift, which moves every TMEM
// lane's data to the lane below it -- inside each 32-lane quarter (the last
// lane of a quarter keeps its data).  So the 128 TMEM lanes hold four bands
// of 32 plane rows that overlap by 2R rows (band g: plane rows VB g .. VB g
// + 31, VB = 32 - 2R); after ky shifts lane 32g + l holds plane row VB g + l
// + ky, exact for l < VB.  A tile therefore has TH = 4 VB output rows (112
// for 5 x 5 filters); 2R rows of each band overlap are staged twice.  Per
// channel: 4 (2R + 1) MMAs of 128 x 16 x 32 (B, 512 bytes per ky, built
// once per CTA, from shared memory) and 3 x 2R shifts of 8 columns; 12
// accumulators (192 TMEM columns).  Shared memory carries only the raw
// input rows, the B slices and the staged output rows.
//
// Interleaved form, R <= 2 (the reference's own runs use 5 x 5): the MMAs
// read the RGB bytes as they lie in the row, with no planes.  Output byte
// o = 3j + c of a row (pixel j, channel c, reading input byte 2 - c) is
//   sum_kx f[ky][kx] * in[o - 2c + 2 + 3 (kx - R)],
// so for the 16 output bytes 16t .. 16t + 15 the inputs lie in the 32-byte
// window 16t - 8 .. 16t + 23 (19 + 6R <= 32 bytes) and
//   B_{ky,ph}[k][n] = f[ky][kx]  where k = n - 2c + 3 (kx - R) + 10, c = (ph + n) % 3,
// with ph = t mod 3 (16 = 1 mod 3): three slices per filter row.  A tile is
// then 12 (2R + 1) MMAs on ONE operand slot of 52 columns (input bytes
// 3 tile_c0 - 8 .. 3 tile_c0 + 199, copied from the raw row unchanged) and
// 7 x 2R shifts; the accumulator columns are the output bytes in order, so
// the epilogue packs four sums to a word with no re-interleave.  The staging
// threads only copy, and the operand slot is double-buffered per tile.
//
// Persistent and warp-specialised: one CTA per SM walks a contiguous range
// of the launch's tiles (horizontal neighbours back to back, so their shared
// input columns are L2 hits).  Ten warps in four roles:
//  - loader (warp 8, one lane): loads the tile's input -- 96+ pixels
//    (tile_c0-16 ..) of TH + 2R rows of the bottom-up image -- as ONE 2-D
//    TMA box (304-byte rows, a tensor map per distinct image) into a ring of
//    raw buffers (2 to 4 slots, as shared memory allows), up to SLOTS tiles
//    ahead.  Views a tensor map cannot describe (not a whole-row NATURAL
//    view, unaligned, or more distinct images than maps) are staged by the
//    staging warps with plain loads;
//  - staging (warps 4-7, TMEM lane quarter = warp - 4): replace rows and
//    pixels beyond the image (TMA fills them with zeros) by the edge row /
//    pixel, then de-interleave thread st's band row by byte permutes and
//    store its three channels into a ring of five TMEM operand slots;
//  - MMA (warp 9, one elected lane): per channel issues the MMAs and shifts
//    on the operand slot into one of two accumulator sets;
//  - epilogue (warps 0-3, TMEM lane quarter = warp): reads its row's 3 x 64
//    sums, packs them to bytes (clamp: saturate; wrap: low byte),
//    re-interleaves RGB into a staged row, frees the accumulator set, and
//    each warp writes its own rows out with coalesced 16-byte stores.
// mbarriers order the roles (raw buffer filled / drained, operands written,
// operand slot consumed, MMAs done = accumulators readable, accumulators
// drained).  Every wait is bounded; a wait that expires sets
// the error word and the CTA stops, waiting (bounded) for its own copies
// and MMAs before it frees its tensor memory.  Reads outside the
// subscription but inside the image's rows (NATURAL views hold whole rows)
// only meet zero filter weights.
constexpr int kTcTW = 64;
constexpr int kTcThreads = 320;     // warps 0-3 epilogue, 4-7 staging, 8 loader, 9 MMA
constexpr int kTcStageWarp0 = 4, kTcLoaderWarp = 8, kTcMmaWarp = 9;
constexpr int kTcMaxR = 8;
constexpr int kTcMaxKD = 2 * kTcMaxR + 1;
constexpr int kTcChunks = 5;        // plane columns tile_c0-8 .. tile_c0+71 in 16-byte chunks (4 TMEM columns each)
constexpr int kRawStride = 304;     // raw row (a TMA box row): pixels tile_c0-16 .. ; 19 x 16 B (odd: conflict-free)
constexpr int kImgfMaps = 4;        // distinct images with a tensor map per launch
constexpr int kOutStride = 208;     // staged output row: 192 B + padding (conflict-free 16-B stores)
// Tensor memory: two accumulator sets of 192 columns (tile k in set k & 1,
// channel c at 64 c) and a ring of five 24-column operand slots (channel
// unit u = 3 k + c in slot u % 5; 5 chunks x 4 columns, shifted in 8-column
// steps).
constexpr uint32_t kTcTmemCols = 512;
constexpr uint32_t kTcAccCols = 192, kTcOpCol0 = 2 * kTcAccCols, kTcOpCols = 24, kTcOpSlots = 5;
static_assert(kTcOpCol0 + kTcOpSlots * kTcOpCols <= kTcTmemCols && 4 * kTcChunks <= kTcOpCols, "tensor memory");
// Interleaved form (R <= kTcIlMaxR): one operand slot per tile, double
// buffered: raw bytes 40 .. 247 of each band row (input bytes 3 tile_c0 - 8 ..
// 3 tile_c0 + 199) in 52 columns, shifted as 7 groups of 8.  Output bytes
// 16 t .. 16 t + 15 read columns 4 t .. 4 t + 7.
constexpr int kTcIlMaxR = 2;
constexpr uint32_t kTcIlOpCols = 56, kTcIlUsedCols = 52;
static_assert(kTcOpCol0 + 2 * kTcIlOpCols <= kTcTmemCols && kTcIlOpCols % 8 == 0 && kTcIlUsedCols <= kTcIlOpCols,
              "tensor memory (interleaved)");
constexpr uint32_t kTcWaitPolls = 1u << 21;
constexpr uint32_t kImgfErrTimeout = 1;
constexpr int kSmemLimit = 227 * 1024 - 256;  // per-block opt-in limit, less the kernel's static shared memory

template <int R>
struct TcGeo {
    static constexpr int KD = 2 * R + 1;
    // R <= 2: the MMAs read the interleaved RGB bytes (no planes), with one
    // banded filter slice per filter row and output-byte phase (16 t mod 3).
    static constexpr bool IL = R <= kTcIlMaxR;
    static constexpr int NB = (IL ? 3 : 1) * KD * 512;   // filter slices in shared memory
    static constexpr int VB = 32 - 2 * R;             // output rows per 32-lane band
    static constexpr int TH = 4 * VB;                 // output rows per tile
    static constexpr int ROWS = TH + 2 * R;           // input rows per tile (TMA box rows)
    static constexpr int RAW = (ROWS * kRawStride + 127) / 128 * 128;  // slot stride (TMA destinations 128-B aligned)
    static constexpr int OUT = TH * kOutStride;
    static constexpr int OFF_RAW = 0;
    static constexpr int FIXED = OFF_RAW + OUT + NB + 256;
    static constexpr int SLOTS = FIXED + 4 * RAW <= kSmemLimit ? 4 : (FIXED + 3 * RAW <= kSmemLimit ? 3 : 2);
    static constexpr int OFF_OUT = OFF_RAW + SLOTS * RAW;
    static constexpr int OFF_B = OFF_OUT + OUT;
    static constexpr int OFF_BAR = OFF_B + NB;
    static constexpr int SMEM = OFF_BAR + 256;
    static_assert(RAW % 128 == 0 && OFF_OUT % 16 == 0 && OFF_B % 16 == 0 &&
                      OFF_BAR % 8 == 0,
                  "alignment");
    static_assert(VB >= 16, "band");
    static_assert(SMEM <= kSmemLimit, "shared memory");
};

// Instruction descriptor, kind::i8: S32 accumulator, A u8, B s8, both
// K-major, N = 16, M = 128.
constexpr uint32_t kTcIdesc = (2u << 4) | (0u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

template <int MAXI>
struct ImgfParamsTc {
    CUtensorMap maps[kImgfMaps];  // the input images (u32 elements, 76 x (TH + 2R) boxes)
    int map_of[MAXI];             // tensor map of each item, -1: plain loads
    int8_t f[kTcMaxKD][kTcMaxKD];
    int n_items;
    int total_tiles;
    int tile_start[MAXI + 1];
    int tiles_x[MAXI];
    uint32_t* err;
    pmb_imgf_item items[MAXI];
};

__device__ __forceinline__ uint32_t tc_smem(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory descriptor of a K-major tile without swizzle: 8-row core
// groups `sbo` bytes apart, 16-byte K chunks `lbo` bytes apart.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFF);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32;
    d |= static_cast<uint64_t>(1) << 46;  // descriptor version (sm_100); layout 0 = no swizzle
    return d;
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kTcWaitPolls; ++i) {
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

__device__ __forceinline__ void tc_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// A from tensor memory ([a] = TMEM address of the 128 x 32-byte operand).
__device__ __forceinline__ void tc_mma_i8_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate)
        : "memory");
}

// Every lane of the 8 columns at taddr takes the data of the lane above it
// (lane + 1) within its 32-lane quarter; the quarter's last lane keeps its own.
__device__ __forceinline__ void tc_shift(uint32_t taddr) {
    asm volatile("tcgen05.shift.cta_group::1.down [%0];" ::"r"(taddr) : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// One lane of the (converged) warp: the one that issues the MMAs.
__device__ __forceinline__ bool tc_elect() {
    uint32_t pred = 0;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "elect.sync _|P, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(pred));
    return pred != 0;
}

// Barrier among the 128 staging threads (id 2).
__device__ __forceinline__ void role_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

__device__ __forceinline__ void tc_st8(uint32_t taddr, const uint32_t (&v)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]),
                 "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}
__device__ __forceinline__ void tc_st4(uint32_t taddr, const uint32_t (&v)[4]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr), "r"(v[0]), "r"(v[1]),
                 "r"(v[2]), "r"(v[3])
                 : "memory");
}

// Chunks Q0 .. Q0 + NQ - 1 of one input row into the warp's TMEM lanes: raw
// bytes 48 q + 24 .. 48 q + 71 hold chunk q (16 pixels); the 16-byte loads
// start at raw byte 48 Q0 + 16 (src points at raw byte 16 of the row).
// Chunk q of channel c goes to columns 4 q .. 4 q + 3 of op[c].  Warp-wide:
// every lane of the warp calls it.
template <int Q0, int NQ>
__device__ __forceinline__ void stage_chunks(const uint8_t* src, const uint32_t (&op)[3]) {
    constexpr int kLoads = (48 * NQ + 8 + 15) / 16;
    uint32_t w[4 * kLoads];
#pragma unroll
    for (int j = 0; j < kLoads; ++j) {
        const uint4 v = *reinterpret_cast<const uint4*>(src + 48 * Q0 + 16 * j);
        w[4 * j] = v.x;
        w[4 * j + 1] = v.y;
        w[4 * j + 2] = v.z;
        w[4 * j + 3] = v.w;
    }
    uint32_t o[3][4 * NQ];
#pragma unroll
    for (int qq = 0; qq < NQ; ++qq)
#pragma unroll
        for (int g = 0; g < 4; ++g)
            deinterleave4(w[12 * qq + 2 + 3 * g], w[12 * qq + 3 + 3 * g], w[12 * qq + 4 + 3 * g], o[0][4 * qq + g],
                          o[1][4 * qq + g], o[2][4 * qq + g]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const uint32_t col = op[c] + 4 * Q0;
        if constexpr (NQ >= 2) {
            const uint32_t v[8] = {o[c][0], o[c][1], o[c][2], o[c][3], o[c][4], o[c][5], o[c][6], o[c][7]};
            tc_st8(col, v);
        }
        if constexpr (NQ == 3) {
            const uint32_t v[4] = {o[c][8], o[c][9], o[c][10], o[c][11]};
            tc_st4(col + 8, v);
        }
    }
}

struct TcTile {
    int item, r0, c0, tw, rows;
    int map;  // tensor map that stages the tile, -1: plain loads
};

// Walks a CTA's contiguous tile range, one tile after the other: tile g of
// the launch lies in item `cur` (tile_start[cur] <= g < tile_start[cur + 1]).
// The item's description is kept in registers and reloaded only when the
// walk enters the next item, so a step costs a few register operations, not
// a chain of dependent loads from the parameter space.
template <int MAXI, int TH>
struct TcCursor {
    int cur, g, end_g, tx, ty, txs, map;
    pmb_imgf_item it;
    __device__ __forceinline__ void enter(const ImgfParamsTc<MAXI>& p) {
        it = p.items[cur];
        txs = p.tiles_x[cur];
        end_g = p.tile_start[cur + 1];
        map = p.map_of[cur];
    }
    __device__ __forceinline__ TcCursor(const ImgfParamsTc<MAXI>& p, int g0) : g(g0) {
        int lo = 0, hi = p.n_items - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.tile_start[mid] <= g0) lo = mid; else hi = mid - 1;
        }
        cur = lo;
        enter(p);
        const int local = g0 - p.tile_start[cur];
        ty = local / txs;
        tx = local - ty * txs;
    }
    __device__ __forceinline__ void next(const ImgfParamsTc<MAXI>& p) {
        ++g;
        if (++tx == txs) {
            tx = 0;
            ++ty;
        }
        if (g >= end_g && cur + 1 < p.n_items) {
            ++cur;  // every item of the launch has at least one tile
            enter(p);
            tx = ty = 0;
        }
    }
    __device__ __forceinline__ TcTile tile() const {
        TcTile t;
        t.item = cur;
        t.c0 = it.c0 + tx * kTcTW;
        t.r0 = it.r0 + ty * TH;
        t.tw = min(kTcTW, it.c1 - t.c0);
        t.rows = min(TH, it.r1 - t.r0);
        t.map = map;
        return t;
    }
};

template <int R, int MODE, int MAXI>
__global__ void __launch_bounds__(kTcThreads, 1)
imgf_tc_kernel(const __grid_constant__ ImgfParamsTc<MAXI> p) {
    using G = TcGeo<R>;
    constexpr int SLOTS = G::SLOTS;
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* const raws = smem + G::OFF_RAW;
    uint8_t* const ost = smem + G::OFF_OUT;
    uint8_t* const bsm = smem + G::OFF_B;
    uint64_t* const bars = reinterpret_cast<uint64_t*>(smem + G::OFF_BAR);
    uint64_t* const full = bars;              // [SLOTS]: raw buffer filled
    uint64_t* const raw_free = bars + 4;      // [SLOTS]: raw buffer drained (4 staging warps)
    uint64_t* const op_full = bars + 8;       // [2]: operands of tile k (k & 1) written (4 staging warps)
    uint64_t* const mma_done = bars + 10;     // [2]: accumulator set written
    uint64_t* const acc_free = bars + 12;     // [2]: accumulator set drained (4 epilogue warps)
    uint64_t* const op_free = bars + 14;      // [5]: operand slot consumed by its unit's MMAs and shifts
    uint64_t* const teardown = bars + 19;
    uint32_t* const tmem_slot = reinterpret_cast<uint32_t*>(bars + 20);
    __shared__ volatile int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // This CTA's tiles: [t_begin, t_end) of the launch, in order.
    const int t_begin = static_cast<int>(static_cast<int64_t>(blockIdx.x) * p.total_tiles / gridDim.x);
    const int t_end = static_cast<int>(static_cast<int64_t>(blockIdx.x + 1) * p.total_tiles / gridDim.x);
    const int ntiles = t_end - t_begin;

    if (tid == 0) {
        s_fail = 0;
        for (int i = 0; i < SLOTS; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&full[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(tc_smem(&raw_free[i])));
        }
        for (int i = 0; i < static_cast<int>(kTcOpSlots); ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&op_free[i])));
        for (int i = 0; i < 2; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(tc_smem(&op_full[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&mma_done[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(tc_smem(&acc_free[i])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(teardown)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // B: per filter row, the 16 x 32 banded slice, K-major core matrices
    // (8 output columns x 16 bytes; column groups 128 B, K chunks 256 B apart).
    // B: per filter row (and, interleaved, per output-byte phase ph), the
    // 16 x 32 banded slice, K-major core matrices (8 output columns x 16
    // bytes; column groups 128 B, K chunks 256 B apart): byte (k, n) at
    // (k / 16) 256 + (n / 8) 128 + (n % 8) 16 + k % 16.  Zeroed, then each
    // tap placed: planar, output column n reads plane column k = n + kx - R + 8
    // of its window; interleaved, output byte n (channel c = (ph + n) % 3)
    // reads window byte k = n - 2c + 3 (kx - R) + 10.
    for (int w = tid; w < G::NB / 4; w += kTcThreads) reinterpret_cast<uint32_t*>(bsm)[w] = 0;
    __syncthreads();
    for (int e = tid; e < (G::NB / 512) * 16 * G::KD; e += kTcThreads) {
        const int kx = e % G::KD, n = (e / G::KD) & 15, slice = e / (16 * G::KD);
        const int ky = G::IL ? slice / 3 : slice;
        const int k = G::IL ? n - 2 * ((slice % 3 + n) % 3) + 3 * (kx - R) + 10 : n + kx - R + 8;
        bsm[slice * 512 + (k >> 4) * 256 + (n >> 3) * 128 + (n & 7) * 16 + (k & 15)] =
            static_cast<uint8_t>(p.f[ky][kx]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == kTcMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(tmem_slot)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    // Launched as a programmatic dependent of the stream's previous kernel:
    // the set-up above (barriers, filter slices, tensor memory) overlaps that
    // kernel's tail, and global memory is touched only from here on, once
    // that kernel is complete and its writes are visible.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    if (warp == kTcLoaderWarp) {
        // ================= loader =================
        // Tile k goes to raw slot k % SLOTS once the staging warps have
        // drained the slot's previous tile.  Box row j holds buffer row
        // y + j, i.e. image row t.r0 - R + ROWS - 1 - j.
        if (lane == 0) {
            TcCursor<MAXI, G::TH> cur(p, t_begin);
            int issued = 0;
            for (; issued < ntiles; ++issued) {
                const int k = issued, s = k % SLOTS;
                if (k > 0) cur.next(p);
                if (s_fail) break;
                if (k >= SLOTS && !tc_wait(tc_smem(&raw_free[s]), ((k / SLOTS) - 1) & 1)) {
                    s_fail = 1;
                    break;
                }
                const TcTile t = cur.tile();
                const uint32_t bar = tc_smem(&full[s]);
                if (t.map < 0) {
                    tc_arrive(bar);  // staged by the staging warps' own loads
                    continue;
                }
                const pmb_imgf_item& it = cur.it;
                const int x = 3 * (t.c0 - 16) / 4;                          // u32 elements; 16-byte multiple
                const int y = it.height - 1 - (t.r0 - R + G::ROWS - 1);     // may be negative: zero-filled rows
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                             "r"(static_cast<uint32_t>(G::ROWS * kRawStride))
                             : "memory");
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                    "[%4];" ::"r"(tc_smem(raws + s * G::RAW)),
                    "l"(reinterpret_cast<uint64_t>(&p.maps[t.map])), "r"(x), "r"(y), "r"(bar)
                    : "memory");
            }
            // After a failure, copies still in flight must land before the
            // CTA's shared memory is released: the last tile issued to each
            // slot completes the slot's latest phase.
            if (s_fail)
                for (int k = max(0, issued - SLOTS); k < issued; ++k) tc_wait(tc_smem(&full[k % SLOTS]), (k / SLOTS) & 1);
        }
    } else if (warp == kTcMmaWarp) {
        // ================= MMA issue =================
        const uint64_t bdesc0 = tc_desc(tc_smem(bsm), 256, 128);
        for (int k = 0; k < ntiles; ++k) {
            if (__any_sync(0xffffffffu, s_fail != 0)) break;
            const int b = k & 1;
            bool ok = tc_wait(tc_smem(&op_full[b]), (k >> 1) & 1);
            // Accumulator set b is free once the epilogue has drained tile k - 2.
            if (ok && k >= 2) ok = tc_wait(tc_smem(&acc_free[b]), ((k - 2) >> 1) & 1);
            if (!__all_sync(0xffffffffu, ok)) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (G::IL && tc_elect()) {
                // Interleaved: 12 output-byte groups per filter row, all on the
                // tile's operand slot; one shift of the slot per filter row.
                const uint32_t op = tmem + kTcOpCol0 + kTcIlOpCols * static_cast<uint32_t>(k & 1);
                const uint32_t acc = tmem + kTcAccCols * b;
#pragma unroll
                for (int ky = 0; ky < G::KD; ++ky) {
#pragma unroll
                    for (int tg = 0; tg < 12; ++tg)
                        tc_mma_i8_ta(acc + 16 * tg, op + 4 * tg,
                                     bdesc0 + static_cast<uint64_t>(((3 * ky + tg % 3) * 512) >> 4), ky > 0 ? 1u : 0u);
                    if (ky + 1 < G::KD) {
#pragma unroll
                        for (uint32_t sc = 0; sc < kTcIlOpCols; sc += 8) tc_shift(op + sc);
                    }
                }
                tc_commit(tc_smem(&op_free[k & 1]));
                tc_commit(tc_smem(&mma_done[b]));
            } else if (!G::IL && tc_elect()) {
#pragma unroll 1
                for (int c = 0; c < 3; ++c) {
                    const int u = 3 * k + c;
                    const uint32_t op = tmem + kTcOpCol0 + kTcOpCols * static_cast<uint32_t>(u % kTcOpSlots);
                    const uint32_t acc = tmem + kTcAccCols * b + 64u * c;
#pragma unroll
                    for (int ky = 0; ky < G::KD; ++ky) {
#pragma unroll
                        for (int tg = 0; tg < 4; ++tg)
                            tc_mma_i8_ta(acc + 16 * tg, op + 4 * tg, bdesc0 + static_cast<uint64_t>((ky * 512) >> 4),
                                         ky > 0 ? 1u : 0u);
                        if (ky + 1 < G::KD) {
                            tc_shift(op);
                            tc_shift(op + 8);
                            tc_shift(op + 16);
                        }
                    }
                    tc_commit(tc_smem(&op_free[u % kTcOpSlots]));
                }
                tc_commit(tc_smem(&mma_done[b]));
            }
            __syncwarp();
        }
    } else if (warp >= kTcStageWarp0) {
        // ================= staging =================
        const int st = tid - 32 * kTcStageWarp0;  // 0..127
        TcCursor<MAXI, G::TH> cur(p, t_begin);
        for (int k = 0; k < ntiles; ++k) {
            if (k > 0) cur.next(p);
            const TcTile t = cur.tile();
            const pmb_imgf_item& it = cur.it;
            const int s = k % SLOTS;
            uint8_t* raw = raws + s * G::RAW;
            // After a failure (s_fail) a staging warp stops waiting and stops
            // working, but keeps walking the tiles and taking part in the role's
            // barriers, so the other staging warps never wait for it there.
            bool ok = s_fail == 0 && tc_wait(tc_smem(&full[s]), (k / SLOTS) & 1);
            const int mlo = max(0, it.r0 - R), mhi = min(it.height - 1, it.r1 - 1 + R);
            const int clo = max(0, it.c0 - R), chi = min(it.width - 1, it.c1 - 1 + R);
            const bool top = t.r0 - R < 0, bottom = t.r0 - R + G::ROWS > it.height;
            const bool left = t.c0 < 16, right = t.c0 + 80 + R > it.width + 16;
            // Raw rows written by the staging threads themselves (plain loads, edge
            // fills) need a role barrier before other threads read them; rows that
            // only TMA wrote are visible to every thread after its own wait.
            const bool shared_writes = t.map < 0 || left || right || top || bottom;
            if (t.map < 0) {
                // Plain loads of the needed pixels, clamped to the subscription.
                const int span = kTcTW + 2 * R;
                for (int e = st; e < G::ROWS * span; e += 128) {
                    const int r = e / span, x = 16 - R + (e - r * span);
                    const int m = pmb::clampi(t.r0 - R + r, mlo, mhi);
                    const int n = pmb::clampi(t.c0 - 16 + x, clo, chi);
                    const uint8_t* src = it.in + static_cast<int64_t>(it.height - 1 - m - it.in_row0) * it.in_pitch +
                                         3 * (n - it.in_col0);
                    uint8_t* d = raw + (G::ROWS - 1 - r) * kRawStride + 3 * x;
                    d[0] = __ldg(src);
                    d[1] = __ldg(src + 1);
                    d[2] = __ldg(src + 2);
                }
            } else {
                if (left || right) {
                    // Needed pixels (x in [16 - R, 80 + R)) beyond the image's left or
                    // right edge -- the halo, or the part of a tile that overhangs
                    // the image -- repeat the edge pixel.
                    const int x0 = max(0, 16 - t.c0), x1 = min(96, it.width - t.c0 + 16);
                    const int nl = max(0, x0 - (16 - R)), nr = max(0, 80 + R - x1), nx = nl + nr;
                    for (int e = st; e < G::ROWS * nx; e += 128) {
                        const int j = e / nx, k2 = e - j * nx;
                        const int x = k2 < nl ? 16 - R + k2 : x1 + (k2 - nl);
                        const int xs = x < x0 ? x0 : x1 - 1;
                        uint8_t* row = raw + j * kRawStride;
                        row[3 * x] = row[3 * xs];
                        row[3 * x + 1] = row[3 * xs + 1];
                        row[3 * x + 2] = row[3 * xs + 2];
                    }
                }
                if (top || bottom) {
                    // The R rows beyond the image's top or bottom repeat the edge
                    // row; rows further out feed only output rows outside the
                    // image, which are not written.
                    role_sync(2);  // edge pixels of the edge rows are in place
                    const int j_top = t.r0 - R + G::ROWS - 1;             // box row of image row 0
                    const int j_bot = t.r0 - R + G::ROWS - it.height;     // box row of image row H - 1
                    const int nt = top ? min(R, G::ROWS - 1 - j_top) : 0;  // box rows j_top + 1 .. j_top + nt
                    const int nb = bottom ? min(R, j_bot) : 0;             // box rows j_bot - nb .. j_bot - 1
                    constexpr int kV = kRawStride / 16;
                    for (int e = st; e < (nt + nb) * kV; e += 128) {
                        const int i = e / kV, v = e - i * kV;
                        const int j = i < nt ? j_top + 1 + i : j_bot - nb + (i - nt);
                        const int js = i < nt ? j_top : j_bot;
                        *reinterpret_cast<uint4*>(raw + j * kRawStride + 16 * v) =
                            *reinterpret_cast<const uint4*>(raw + js * kRawStride + 16 * v);
                    }
                }
            }
            if (G::IL) {
                // The tile's operand slot is free once tile k - 2's MMAs and shifts are done.
                if (k >= 2) ok = ok && tc_wait(tc_smem(&op_free[k & 1]), ((k >> 1) - 1) & 1);
            } else {
                // Operand slot of unit u = 3k + c is free once the MMAs and shifts of
                // unit u - 5 are done.
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int u = 3 * k + c;
                    if (u >= static_cast<int>(kTcOpSlots))
                        ok = ok &&
                             tc_wait(tc_smem(&op_free[u % kTcOpSlots]), ((u / static_cast<int>(kTcOpSlots)) - 1) & 1);
                }
            }
            ok = __all_sync(0xffffffffu, ok);
            if (shared_writes) role_sync(2);  // raw rows complete (loads and edge fills)
            if (!ok) {
                s_fail = 1;
                continue;
            }
            // De-interleave: thread st stages band row st (band st / 32, plane row
            // VB (st / 32) + st % 32) into TMEM lane st of the three operand
            // slots.  Consecutive threads take consecutive rows, so the 16-byte
            // loads (row stride 19 x 16 B) are conflict-free.
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (G::IL) {
                // Interleaved: raw bytes 40 .. 247 of band row st, as they are,
                // into TMEM lane st of the tile's slot (16-byte loads from raw
                // byte 32; words 2 .. 53 go to columns 0 .. 51).
                const int r = G::VB * (st >> 5) + (st & 31);
                const uint4* const src = reinterpret_cast<const uint4*>(raw + (G::ROWS - 1 - r) * kRawStride + 32);
                const uint32_t col0 = tmem + (static_cast<uint32_t>(st & ~31) << 16) + kTcOpCol0 +
                                      kTcIlOpCols * static_cast<uint32_t>(k & 1);
                // Two rounds (loads 0-7, then 8-13) keep fewer words live.
                uint32_t w[56];
#pragma unroll
                for (int half = 0; half < 2; ++half) {
#pragma unroll
                    for (int j = 8 * half; j < (half ? 14 : 8); ++j) {
                        const uint4 v = src[j];
                        w[4 * j] = v.x;
                        w[4 * j + 1] = v.y;
                        w[4 * j + 2] = v.z;
                        w[4 * j + 3] = v.w;
                    }
#pragma unroll
                    for (int g = 3 * half; g < (half ? 6 : 3); ++g) {
                        const uint32_t v[8] = {w[8 * g + 2], w[8 * g + 3], w[8 * g + 4], w[8 * g + 5],
                                               w[8 * g + 6], w[8 * g + 7], w[8 * g + 8], w[8 * g + 9]};
                        tc_st8(col0 + 8 * g, v);
                    }
                }
                const uint32_t v4[4] = {w[50], w[51], w[52], w[53]};
                tc_st4(col0 + 48, v4);
            } else {
                const int r = G::VB * (st >> 5) + (st & 31);
                const uint8_t* const src = raw + (G::ROWS - 1 - r) * kRawStride + 16;
                const uint32_t lanes = tmem + (static_cast<uint32_t>(st & ~31) << 16);
                uint32_t op[3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    op[c] = lanes + kTcOpCol0 + kTcOpCols * static_cast<uint32_t>((3 * k + c) % kTcOpSlots);
                stage_chunks<0, 3>(src, op);  // raw bytes 16 .. 175
                stage_chunks<3, 2>(src, op);  // raw bytes 160 .. 271
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                tc_arrive(tc_smem(&op_full[k & 1]));
                tc_arrive(tc_smem(&raw_free[s]));
            }
        }
    } else {
        // ================= epilogue =================
        // Lane l < VB of quarter q holds output row VB q + l of the tile.
        const int q = warp, row = G::VB * q + lane;
        const bool valid_lane = lane < G::VB;
        TcCursor<MAXI, G::TH> cur(p, t_begin);
        for (int k = 0; k < ntiles; ++k) {
            if (k > 0) cur.next(p);
            const TcTile t = cur.tile();
            const pmb_imgf_item& it = cur.it;
            const int b = k & 1;
            // Each epilogue warp decides for itself (no role barrier follows).
            if (!__all_sync(0xffffffffu, s_fail == 0 && tc_wait(tc_smem(&mma_done[b]), (k >> 1) & 1))) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint8_t* const ostb = ost;
            uint8_t* const orow = ostb + row * kOutStride;
            if constexpr (G::IL) {
                // Interleaved: accumulator column 16 t + n is output byte 16 t + n
                // of the row, so four sums pack into a word in place.
                uint32_t pw[48];
#pragma unroll
                for (int h = 0; h < 3; ++h) {
                    uint32_t v[4][16];
#pragma unroll
                    for (int tg = 0; tg < 4; ++tg)
                        tc_ld16(tmem + kTcAccCols * b + (static_cast<uint32_t>(32 * q) << 16) +
                                    static_cast<uint32_t>(64 * h + 16 * tg),
                                v[tg]);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int tg = 0; tg < 4; ++tg)
#pragma unroll
                        for (int g = 0; g < 4; ++g) {
                            const int a[4] = {static_cast<int>(v[tg][4 * g]), static_cast<int>(v[tg][4 * g + 1]),
                                              static_cast<int>(v[tg][4 * g + 2]), static_cast<int>(v[tg][4 * g + 3])};
                            pw[16 * h + 4 * tg + g] = pack4<MODE>(a);
                        }
                }
                // The accumulator set is drained: the MMAs of tile k + 2 may start.
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) tc_arrive(tc_smem(&acc_free[b]));
                if (valid_lane) {
#pragma unroll
                    for (int i = 0; i < 12; ++i)
                        *reinterpret_cast<uint4*>(orow + 16 * i) =
                            make_uint4(pw[4 * i], pw[4 * i + 1], pw[4 * i + 2], pw[4 * i + 3]);
                }
            } else {
                uint32_t pw[3][16];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    uint32_t v[4][16];
#pragma unroll
                    for (int tg = 0; tg < 4; ++tg)
                        tc_ld16(tmem + kTcAccCols * b + (static_cast<uint32_t>(32 * q) << 16) +
                                    static_cast<uint32_t>(64 * c + 16 * tg),
                                v[tg]);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int tg = 0; tg < 4; ++tg)
#pragma unroll
                        for (int g = 0; g < 4; ++g) {
                            const int a[4] = {static_cast<int>(v[tg][4 * g]), static_cast<int>(v[tg][4 * g + 1]),
                                              static_cast<int>(v[tg][4 * g + 2]), static_cast<int>(v[tg][4 * g + 3])};
                            pw[c][4 * tg + g] = pack4<MODE>(a);
                        }
                }
                // The accumulator set is drained: the MMAs of tile k + 2 may start.
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) tc_arrive(tc_smem(&acc_free[b]));
#pragma unroll
                for (int g = 0; g < (valid_lane ? 16 : 0); g += 4) {
                    uint32_t d[12];
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const uint32_t A = pw[0][g + h], B = pw[1][g + h], C = pw[2][g + h];
                        d[3 * h + 0] = __byte_perm(__byte_perm(A, B, 0x0140), C, 0x2410);  // a0 b0 c0 a1
                        d[3 * h + 1] = __byte_perm(__byte_perm(B, C, 0x0251), A, 0x2610);  // b1 c1 a2 b2
                        d[3 * h + 2] = __byte_perm(C, __byte_perm(A, B, 0x0073), 0x3542);  // c2 a3 b3 c3
                    }
#pragma unroll
                    for (int h = 0; h < 3; ++h)
                        *reinterpret_cast<uint4*>(orow + 12 * g + 16 * h) =
                            make_uint4(d[4 * h], d[4 * h + 1], d[4 * h + 2], d[4 * h + 3]);
                }
            }
            // Each warp writes out the rows it staged (tile rows VB q .. VB q +
            // VB - 1): 12 16-byte pieces per row, consecutive lanes on
            // consecutive pieces.  Only the warp's own rows are read, so a warp
            // barrier orders the staging and the copy, and the next tile's
            // staging of the same rows comes after this copy in program order.
            __syncwarp();
            const int r_lo = G::VB * q, r_hi = min(r_lo + G::VB, t.rows);
            uint8_t* const obase = it.out + static_cast<int64_t>(t.r0 - it.out_row0) * it.out_pitch +
                                   3 * (t.c0 - it.out_col0);
            if (t.tw == kTcTW && ((reinterpret_cast<uintptr_t>(obase) | static_cast<uintptr_t>(it.out_pitch)) & 15) == 0) {
                constexpr int kPer = (G::VB * 12 + 31) / 32;
                const int n = (r_hi - r_lo) * 12;
                uint4 v[kPer];
#pragma unroll
                for (int i = 0; i < kPer; ++i) {
                    const int e = lane + 32 * i, r = r_lo + e / 12, c = e % 12;
                    if (e < n) v[i] = *reinterpret_cast<const uint4*>(ostb + r * kOutStride + 16 * c);
                }
#pragma unroll
                for (int i = 0; i < kPer; ++i) {
                    const int e = lane + 32 * i, r = r_lo + e / 12, c = e % 12;
                    if (e < n) *reinterpret_cast<uint4*>(obase + static_cast<int64_t>(r) * it.out_pitch + 16 * c) = v[i];
                }
            } else {
                const int nb = 3 * t.tw;
                for (int e = lane; e < (r_hi - r_lo) * nb; e += 32) {
                    const int r = r_lo + e / nb, c = e % nb;
                    obase[static_cast<int64_t>(r) * it.out_pitch + c] = ostb[r * kOutStride + c];
                }
            }
            __syncwarp();
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == kTcMmaWarp) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (s_fail && tc_elect()) {  // the lane that issued the MMAs
            atomicOr(p.err, kImgfErrTimeout);
            tc_commit(tc_smem(teardown));  // every MMA this CTA issued has retired once this arrives
            tc_wait(tc_smem(teardown), 0);
        }
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Plain GPU form: one thread per output pixel, byte loads straight from HBM.
struct PlainFilter {
    int8_t f[PMB_IMGF_MAX_FILTER_DIM][PMB_IMGF_MAX_FILTER_DIM];
};

template <int MODE>
__global__ void imgf_plain_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int W,
                                  int H, int R, const __grid_constant__ PlainFilter pf) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= W || i >= H) return;
    int s0 = 0, s1 = 0, s2 = 0;
    for (int ky = 0; ky <= 2 * R; ++ky) {
        const int m = pmb::clampi(i + ky - R, 0, H - 1);
        const uint8_t* row = in + static_cast<int64_t>(H - 1 - m) * 3 * W;
        for (int kx = 0; kx <= 2 * R; ++kx) {
            const int n = pmb::clampi(j + kx - R, 0, W - 1);
            const int f = pf.f[ky][kx];
            s0 += row[3 * n + 2] * f;
            s1 += row[3 * n + 1] * f;
            s2 += row[3 * n + 0] * f;
        }
    }
    uint8_t* o = out + (static_cast<int64_t>(i) * W + j) * 3;
    if (MODE == PMB_IMGF_WRAP) {
        o[0] = static_cast<uint8_t>(s0);
        o[1] = static_cast<uint8_t>(s1);
        o[2] = static_cast<uint8_t>(s2);
    } else {
        o[0] = static_cast<uint8_t>(min(max(s0, 0), 255));
        o[1] = static_cast<uint8_t>(min(max(s1, 0), 255));
        o[2] = static_cast<uint8_t>(min(max(s2, 0), 255));
    }
}

// ---------------------------------------------------------------------------
int validate_item(const pmb_imgf_item& it, int R, int idx) {
    PMB_CHECK_ARG(it.in && it.out, "item %d: null pointer", idx);
    PMB_CHECK_ARG(it.width > 0 && it.height > 0, "item %d: bad image size %dx%d", idx, it.width,
                  it.height);
    PMB_CHECK_ARG(0 <= it.r0 && it.r0 <= it.r1 && it.r1 <= it.height && 0 <= it.c0 &&
                      it.c0 <= it.c1 && it.c1 <= it.width,
                  "item %d: rectangle [%d,%d)x[%d,%d) outside %dx%d image", idx, it.r0, it.r1,
                  it.c0, it.c1, it.width, it.height);
    if (it.r0 == it.r1 || it.c0 == it.c1) return PMB_SUCCESS;
    const int mhi = std::min(it.height - 1, it.r1 - 1 + R);
    const int clo = std::max(0, it.c0 - R), chi = std::min(it.width - 1, it.c1 - 1 + R);
    PMB_CHECK_ARG(it.in_row0 >= 0 && it.in_row0 <= it.height - 1 - mhi && it.in_col0 >= 0 &&
                      it.in_col0 <= clo,
                  "item %d: input view origin (%d,%d) does not cover the subscription", idx,
                  it.in_row0, it.in_col0);
    PMB_CHECK_ARG(it.in_pitch >= 3LL * (chi - it.in_col0 + 1), "item %d: input pitch too small",
                  idx);
    PMB_CHECK_ARG(it.out_row0 >= 0 && it.out_row0 <= it.r0 && it.out_col0 >= 0 &&
                      it.out_col0 <= it.c0,
                  "item %d: output view origin does not cover the rectangle", idx);
    PMB_CHECK_ARG(it.out_pitch >= 3LL * (it.c1 - it.out_col0), "item %d: output pitch too small",
                  idx);
    return PMB_SUCCESS;
}

// Pixel (m, n) of an item's input is read at in_base + (H-1-m) * in_pitch + 3n
// and written at out_base + m * out_pitch + 3n: two items with the same
// bases, whole-row pitches and image size address every pixel identically,
// so where their output rectangles are adjacent (same rows and touching
// columns, or same columns and touching rows) one item covering both
// computes the same bytes, and it reads and writes only memory inside the
// two items' views.
struct ItemKey {
    uintptr_t in_base, out_base;
    int width, height;
    bool operator==(const ItemKey& o) const {
        return in_base == o.in_base && out_base == o.out_base && width == o.width && height == o.height;
    }
};

ItemKey key_of(const pmb_imgf_item& it) {
    ItemKey k;
    k.in_base = reinterpret_cast<uintptr_t>(it.in) - static_cast<uintptr_t>(it.in_row0 * it.in_pitch) -
                3u * static_cast<uintptr_t>(it.in_col0);
    k.out_base = reinterpret_cast<uintptr_t>(it.out) - static_cast<uintptr_t>(it.out_row0 * it.out_pitch) -
                 3u * static_cast<uintptr_t>(it.out_col0);
    k.width = it.width;
    k.height = it.height;
    return k;
}

// Merges adjacent items in two sorted passes (rows of touching column
// ranges, then columns of touching row ranges); drops empty rectangles.
// Items with a pitch other than 3W (COMPACT views) are kept as they are.
// Returns the number of items written to `out`.
int coalesce_items(const pmb_imgf_item* items, int n, pmb_imgf_item* out) {
    // Small records sorted in place (no allocation): the item's group of
    // identical keys, its rectangle and its index.
    struct Rect {
        int g, idx, r0, r1, c0, c1;
    };
    Rect e[PMB_IMGF_MAX_ITEMS];
    ItemKey keys[PMB_IMGF_MAX_ITEMS];
    int ne = 0, nk = 0, m = 0;
    for (int i = 0; i < n; ++i) {
        const pmb_imgf_item& it = items[i];
        if (it.r0 == it.r1 || it.c0 == it.c1) continue;
        if (it.in_pitch != 3LL * it.width || it.out_pitch != 3LL * it.width) {
            out[m++] = it;
            continue;
        }
        const ItemKey k = key_of(it);
        int g = 0;
        while (g < nk && !(keys[g] == k)) ++g;
        if (g == nk) keys[nk++] = k;
        e[ne++] = {g, i, it.r0, it.r1, it.c0, it.c1};
    }
    auto merge_pass = [&e, &ne](bool rows) {
        std::sort(e, e + ne, [rows](const Rect& a, const Rect& b) {
            if (a.g != b.g) return a.g < b.g;
            const int a1 = rows ? a.r0 : a.c0, b1 = rows ? b.r0 : b.c0;
            const int a2 = rows ? a.r1 : a.c1, b2 = rows ? b.r1 : b.c1;
            const int a3 = rows ? a.c0 : a.r0, b3 = rows ? b.c0 : b.r0;
            if (a1 != b1) return a1 < b1;
            if (a2 != b2) return a2 < b2;
            return a3 < b3;
        });
        int w = 0;
        for (int i = 0; i < ne; ++i) {
            if (w > 0) {
                Rect& p = e[w - 1];
                const Rect& c = e[i];
                if (p.g == c.g) {
                    if (rows && p.r0 == c.r0 && p.r1 == c.r1 && p.c1 == c.c0) {
                        p.c1 = c.c1;
                        continue;
                    }
                    if (!rows && p.c0 == c.c0 && p.c1 == c.c1 && p.r1 == c.r0) {
                        p.r1 = c.r1;
                        continue;
                    }
                }
            }
            e[w++] = e[i];
        }
        ne = w;
    };
    merge_pass(true);
    merge_pass(false);
    for (int i = 0; i < ne; ++i) {
        pmb_imgf_item it = items[e[i].idx];
        it.r0 = e[i].r0;
        it.r1 = e[i].r1;
        it.c0 = e[i].c0;
        it.c1 = e[i].c1;
        out[m++] = it;
    }
    return m;
}

template <int R, int MODE, int MAXI>
int launch_t(const pmb_imgf_item* items, int n, const int8_t* filter, cudaStream_t s) {
    using G = Geo<R>;
    ImgfParams<R, MAXI> p;
    for (int ky = 0; ky < G::KD; ++ky)
        for (int k = 0; k < 4; ++k)
            for (int w = 0; w < G::NW; ++w) {
                uint32_t word = 0;
                for (int b = 0; b < 4; ++b) {
                    const int kx = 4 * w + b - G::OFF - k;
                    if (kx >= 0 && kx < G::KD)
                        word |= static_cast<uint32_t>(
                                    static_cast<uint8_t>(filter[ky * PMB_IMGF_MAX_FILTER_DIM + kx]))
                                << (8 * b);
                }
                p.pat[ky][k][w] = word;
            }
    int64_t total = 0;
    int m = 0;
    for (int i = 0; i < n; ++i) {
        const pmb_imgf_item& it = items[i];
        if (it.r0 == it.r1 || it.c0 == it.c1) continue;
        const int txs = (it.c1 - it.c0 + kTW - 1) / kTW;
        const int tys = (it.r1 - it.r0 + kTH - 1) / kTH;
        p.items[m] = it;
        p.tiles_x[m] = txs;
        p.tile_start[m] = static_cast<int>(total);
        total += static_cast<int64_t>(txs) * tys;
        ++m;
    }
    if (m == 0) return PMB_SUCCESS;
    if (total > 0x7fffffffLL) return pmb::fail(PMB_BEYOND_LIMITS, "too many tiles: %lld", (long long)total);
    p.n_items = m;
    p.tile_start[m] = static_cast<int>(total);
    imgf_kernel<R, MODE, MAXI><<<static_cast<unsigned>(total), kThreads, 0, s>>>(p);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

// Device address of the stencil's error word on the current device.
__device__ uint32_t g_imgf_err;

int imgf_err_word(uint32_t** out) {
    static std::mutex mu;
    static uint32_t* per_dev[64] = {};
    int dev = 0;
    PMB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return pmb::fail(PMB_BEYOND_LIMITS, "device ordinal %d", dev);
    std::lock_guard<std::mutex> g(mu);
    if (!per_dev[dev]) {
        void* a = nullptr;
        PMB_CUDA_TRY(cudaGetSymbolAddress(&a, g_imgf_err));
        per_dev[dev] = static_cast<uint32_t*>(a);
    }
    *out = per_dev[dev];
    return PMB_SUCCESS;
}

template <int R, int MODE, int MAXI>
int launch_tc(const pmb_imgf_item* items, int n, const int8_t* filter, cudaStream_t s) {
    using G = TcGeo<R>;
    ImgfParamsTc<MAXI> p;
    for (int ky = 0; ky < kTcMaxKD; ++ky)
        for (int kx = 0; kx < kTcMaxKD; ++kx)
            p.f[ky][kx] = ky < G::KD && kx < G::KD ? filter[ky * PMB_IMGF_MAX_FILTER_DIM + kx] : 0;
    int64_t total = 0;
    int m = 0;
    for (int i = 0; i < n; ++i) {
        const pmb_imgf_item& it = items[i];
        if (it.r0 == it.r1 || it.c0 == it.c1) continue;
        const int txs = (it.c1 - it.c0 + kTcTW - 1) / kTcTW;
        const int tys = (it.r1 - it.r0 + G::TH - 1) / G::TH;
        p.items[m] = it;
        p.tiles_x[m] = txs;
        p.tile_start[m] = static_cast<int>(total);
        total += static_cast<int64_t>(txs) * tys;
        ++m;
    }
    if (m == 0) return PMB_SUCCESS;
    if (total > 0x7fffffffLL) return pmb::fail(PMB_BEYOND_LIMITS, "too many tiles: %lld", (long long)total);
    p.n_items = m;
    p.total_tiles = static_cast<int>(total);
    p.tile_start[m] = static_cast<int>(total);
    // Tensor maps: one per distinct image among the items whose view is a
    // whole-row NATURAL view that TMA can address (16-byte aligned image and
    // pitch, whole 16-pixel tile columns); the other items use plain loads.
    int nmaps = 0;
    const uint8_t* bases[kImgfMaps] = {};
    int widths[kImgfMaps] = {}, heights[kImgfMaps] = {};
    pmb::EncodeTiledFn enc = pmb::tensor_map_encoder();
    for (int i = 0; i < m; ++i) {
        const pmb_imgf_item& it = p.items[i];
        p.map_of[i] = -1;
        const uint8_t* base = it.in - it.in_row0 * it.in_pitch - 3 * static_cast<int64_t>(it.in_col0);
        if (!enc || it.in_pitch != 3LL * it.width || (it.width & 3) || (it.c0 & 15) || (it.in_pitch & 15) ||
            (reinterpret_cast<uintptr_t>(base) & 15))
            continue;
        int k = 0;
        while (k < nmaps && !(bases[k] == base && widths[k] == it.width && heights[k] == it.height)) ++k;
        if (k == nmaps) {
            if (nmaps == kImgfMaps) continue;
            const cuuint64_t dims[2] = {static_cast<cuuint64_t>(3 * it.width / 4), static_cast<cuuint64_t>(it.height)};
            const cuuint64_t strides[1] = {static_cast<cuuint64_t>(it.in_pitch)};
            const cuuint32_t box[2] = {kRawStride / 4, static_cast<cuuint32_t>(G::ROWS)};
            const cuuint32_t estr[2] = {1, 1};
            const CUresult r = enc(&p.maps[k], CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint8_t*>(base), dims,
                                   strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) continue;
            bases[k] = base;
            widths[k] = it.width;
            heights[k] = it.height;
            ++nmaps;
        }
        p.map_of[i] = k;
    }
    int st = imgf_err_word(&p.err);
    if (st != PMB_SUCCESS) return st;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(imgf_tc_kernel<R, MODE, MAXI>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
        if (attr == cudaSuccess &&
            pmb::tmem_exclusive(reinterpret_cast<const void*>(imgf_tc_kernel<R, MODE, MAXI>), kTcThreads, G::SMEM,
                                "imgf_tc_kernel") != PMB_SUCCESS)
            attr = cudaErrorInvalidConfiguration;
    });
    PMB_CUDA_TRY(attr);
    int dev = 0, sms = 148;
    PMB_CUDA_TRY(cudaGetDevice(&dev));
    PMB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>(total, sms));  // persistent: one CTA per SM
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kTcThreads);
    cfg.dynamicSmemBytes = G::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute pdl[1];
    pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    pdl[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl;
    cfg.numAttrs = 1;
    PMB_CUDA_TRY(cudaLaunchKernelEx(&cfg, imgf_tc_kernel<R, MODE, MAXI>, p));
    return PMB_SUCCESS;
}

template <int R, int MAXI>
int launch_mode(const pmb_imgf_item* items, int n, const int8_t* filter, int mode, cudaStream_t s) {
    if constexpr (R <= kTcMaxR) {
        return mode == PMB_IMGF_WRAP ? launch_tc<R, PMB_IMGF_WRAP, MAXI>(items, n, filter, s)
                                     : launch_tc<R, PMB_IMGF_CLAMP, MAXI>(items, n, filter, s);
    } else {
        return mode == PMB_IMGF_WRAP ? launch_t<R, PMB_IMGF_WRAP, MAXI>(items, n, filter, s)
                                     : launch_t<R, PMB_IMGF_CLAMP, MAXI>(items, n, filter, s);
    }
}

template <int MAXI>
int launch_radius(const pmb_imgf_item* items, int n, const int8_t* filter, int R, int mode,
                  cudaStream_t s) {
    switch (R) {
#define PMB_IMGF_CASE(r) \
    case r: return launch_mode<r, MAXI>(items, n, filter, mode, s);
        PMB_IMGF_CASE(1) PMB_IMGF_CASE(2) PMB_IMGF_CASE(3) PMB_IMGF_CASE(4) PMB_IMGF_CASE(5)
        PMB_IMGF_CASE(6) PMB_IMGF_CASE(7) PMB_IMGF_CASE(8) PMB_IMGF_CASE(9) PMB_IMGF_CASE(10)
        PMB_IMGF_CASE(11) PMB_IMGF_CASE(12) PMB_IMGF_CASE(13) PMB_IMGF_CASE(14) PMB_IMGF_CASE(15)
#undef PMB_IMGF_CASE
        default: return pmb::fail(PMB_INVALID_INDEX, "filter radius %d outside [1,%d]", R, PMB_IMGF_MAX_RADIUS);
    }
}

}  // namespace

extern "C" int pmb_image_filter(const pmb_imgf_item* items, int n_items, const int8_t* filter,
                                int radius, int mode, void* stream) {
    PMB_CHECK_ARG(items && filter, "null items/filter");
    PMB_CHECK_ARG(n_items >= 1 && n_items <= PMB_IMGF_MAX_ITEMS, "n_items %d outside [1,%d]",
                  n_items, PMB_IMGF_MAX_ITEMS);
    PMB_CHECK_ARG(radius >= 1 && radius <= PMB_IMGF_MAX_RADIUS, "filter radius %d outside [1,%d]",
                  radius, PMB_IMGF_MAX_RADIUS);
    PMB_CHECK_ARG(mode == PMB_IMGF_WRAP || mode == PMB_IMGF_CLAMP, "bad mode %d", mode);
    for (int i = 0; i < n_items; ++i) {
        const int st = validate_item(items[i], radius, i);
        if (st != PMB_SUCCESS) return st;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Subtasks that tile a larger rectangle of the same whole-row views are
    // filtered as that rectangle: same bytes, one tile grid (no partial tiles
    // at the subtask seams) and a smaller launch.
    pmb_imgf_item merged[PMB_IMGF_MAX_ITEMS];
    const int n = coalesce_items(items, n_items, merged);
    return n <= 8 ? launch_radius<8>(merged, n, filter, radius, mode, s)
                  : launch_radius<PMB_IMGF_MAX_ITEMS>(merged, n, filter, radius, mode, s);
}

extern "C" int pmb_image_filter_cover(const pmb_imgf_item* items, int n_items, pmb_imgf_item* out, int* n_out) {
    PMB_CHECK_ARG(items && out && n_out, "null items/out/n_out");
    PMB_CHECK_ARG(n_items >= 1 && n_items <= PMB_IMGF_MAX_ITEMS, "n_items %d outside [1,%d]", n_items,
                  PMB_IMGF_MAX_ITEMS);
    *n_out = coalesce_items(items, n_items, out);
    return PMB_SUCCESS;
}

extern "C" int pmb_image_filter_full(const uint8_t* d_in, uint8_t* d_out, int width, int height,
                                     const int8_t* filter, int radius, int mode, void* stream) {
    pmb_imgf_item it;
    it.in = d_in;
    it.out = d_out;
    it.in_pitch = it.out_pitch = 3LL * width;
    it.width = width;
    it.height = height;
    it.in_row0 = it.in_col0 = it.out_row0 = it.out_col0 = 0;
    it.r0 = 0;
    it.r1 = height;
    it.c0 = 0;
    it.c1 = width;
    return pmb_image_filter(&it, 1, filter, radius, mode, stream);
}

extern "C" int pmb_image_filter_error(int clear, uint32_t* error_out) {
    PMB_CHECK_ARG(error_out, "null pointer");
    uint32_t* w = nullptr;
    const int st = imgf_err_word(&w);
    if (st != PMB_SUCCESS) return st;
    PMB_CUDA_TRY(cudaMemcpy(error_out, w, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (clear) PMB_CUDA_TRY(cudaMemset(w, 0, sizeof(uint32_t)));
    return PMB_SUCCESS;
}

extern "C" int pmb_image_filter_plain(const uint8_t* d_in, uint8_t* d_out, int width, int height,
                                      const int8_t* filter, int radius, int mode, void* stream) {
    PMB_CHECK_ARG(d_in && d_out && filter, "null pointer");
    PMB_CHECK_ARG(width > 0 && height > 0, "bad image size");
    PMB_CHECK_ARG(radius >= 1 && radius <= PMB_IMGF_MAX_RADIUS, "bad radius %d", radius);
    PMB_CHECK_ARG(mode == PMB_IMGF_WRAP || mode == PMB_IMGF_CLAMP, "bad mode %d", mode);
    PlainFilter pf;
    for (int i = 0; i < PMB_IMGF_MAX_FILTER_DIM * PMB_IMGF_MAX_FILTER_DIM; ++i)
        pf.f[i / PMB_IMGF_MAX_FILTER_DIM][i % PMB_IMGF_MAX_FILTER_DIM] = filter[i];
    dim3 block(32, 8);
    dim3 grid((width + 31) / 32, (height + 7) / 8);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (mode == PMB_IMGF_WRAP)
        imgf_plain_kernel<PMB_IMGF_WRAP><<<grid, block, 0, s>>>(d_in, d_out, width, height, radius, pf);
    else
        imgf_plain_kernel<PMB_IMGF_CLAMP><<<grid, block, 0, s>>>(d_in, d_out, width, height, radius, pf);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

// ---------------------------------------------------------------------------
// Host-to-host form: the whole image comes from and returns to host memory.
// Row bands are pipelined over three streams -- band k+1 uploads while band k
// is filtered and band k-1 downloads -- so the PCIe transfers in both
// directions overlap each other and the stencil.  Only the rows a band adds
// (its new rows plus halo not yet uploaded) cross PCIe.
namespace {

struct PipeStreams {
    cudaStream_t up = nullptr, down = nullptr;
};

int pipe_streams(PipeStreams& ps) {
    static std::mutex mu;
    static PipeStreams per_dev[64];
    int dev = 0;
    PMB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return pmb::fail(PMB_BEYOND_LIMITS, "device ordinal %d", dev);
    std::lock_guard<std::mutex> g(mu);
    if (!per_dev[dev].up) {
        PMB_CUDA_TRY(cudaStreamCreateWithFlags(&per_dev[dev].up, cudaStreamNonBlocking));
        PMB_CUDA_TRY(cudaStreamCreateWithFlags(&per_dev[dev].down, cudaStreamNonBlocking));
    }
    ps = per_dev[dev];
    return PMB_SUCCESS;
}

}  // namespace

extern "C" int pmb_image_filter_host(const uint8_t* h_in, uint8_t* h_out, uint8_t* d_in, uint8_t* d_out, int width,
                                     int height, const int8_t* filter, int radius, int mode, int bands, void* stream) {
    PMB_CHECK_ARG(h_in && h_out && d_in && d_out && filter, "null pointer");
    PMB_CHECK_ARG(width > 0 && height > 0, "bad image size");
    PMB_CHECK_ARG(radius >= 1 && radius <= PMB_IMGF_MAX_RADIUS, "filter radius %d outside [1,%d]", radius,
                  PMB_IMGF_MAX_RADIUS);
    PMB_CHECK_ARG(bands >= 1 && bands <= 256, "bands %d outside [1,256]", bands);
    if (bands > height) bands = height;
    PipeStreams ps;
    int st = pipe_streams(ps);
    if (st != PMB_SUCCESS) return st;
    cudaStream_t comp = static_cast<cudaStream_t>(stream);
    const int64_t pitch = 3LL * width;
    const int R = radius;
    // Events are created per call (cheap); recorded ones may be destroyed at once.
    cudaEvent_t start, ev_up[256], ev_k[256], done;
    PMB_CUDA_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    PMB_CUDA_TRY(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    PMB_CUDA_TRY(cudaEventRecord(start, comp));
    PMB_CUDA_TRY(cudaStreamWaitEvent(ps.up, start, 0));
    PMB_CUDA_TRY(cudaStreamWaitEvent(ps.down, start, 0));
    int uploaded_hi = 0;  // image rows [0, uploaded_hi) are on the device
    for (int b = 0; b < bands; ++b) {
        const int r0 = static_cast<int>(static_cast<int64_t>(height) * b / bands);
        const int r1 = static_cast<int>(static_cast<int64_t>(height) * (b + 1) / bands);
        const int need_hi = r1 + R < height ? r1 + R : height;
        if (need_hi > uploaded_hi) {
            // image rows [uploaded_hi, need_hi) = buffer rows [H - need_hi, H - uploaded_hi)
            const int64_t off = static_cast<int64_t>(height - need_hi) * pitch;
            const size_t bytes = static_cast<size_t>(need_hi - uploaded_hi) * pitch;
            PMB_CUDA_TRY(cudaMemcpyAsync(d_in + off, h_in + off, bytes, cudaMemcpyHostToDevice, ps.up));
            uploaded_hi = need_hi;
        }
        PMB_CUDA_TRY(cudaEventCreateWithFlags(&ev_up[b], cudaEventDisableTiming));
        PMB_CUDA_TRY(cudaEventRecord(ev_up[b], ps.up));
        PMB_CUDA_TRY(cudaStreamWaitEvent(comp, ev_up[b], 0));
        pmb_imgf_item it;
        it.in = d_in;
        it.out = d_out;
        it.in_pitch = it.out_pitch = pitch;
        it.width = width;
        it.height = height;
        it.in_row0 = it.in_col0 = it.out_row0 = it.out_col0 = 0;
        it.r0 = r0;
        it.r1 = r1;
        it.c0 = 0;
        it.c1 = width;
        st = pmb_image_filter(&it, 1, filter, radius, mode, comp);
        if (st != PMB_SUCCESS) return st;
        PMB_CUDA_TRY(cudaEventCreateWithFlags(&ev_k[b], cudaEventDisableTiming));
        PMB_CUDA_TRY(cudaEventRecord(ev_k[b], comp));
        PMB_CUDA_TRY(cudaStreamWaitEvent(ps.down, ev_k[b], 0));
        PMB_CUDA_TRY(cudaMemcpyAsync(h_out + static_cast<int64_t>(r0) * pitch, d_out + static_cast<int64_t>(r0) * pitch,
                                     static_cast<size_t>(r1 - r0) * pitch, cudaMemcpyDeviceToHost, ps.down));
    }
    PMB_CUDA_TRY(cudaEventRecord(done, ps.down));
    PMB_CUDA_TRY(cudaStreamWaitEvent(comp, done, 0));
    for (int b = 0; b < bands; ++b) {
        cudaEventDestroy(ev_up[b]);
        cudaEventDestroy(ev_k[b]);
    }
    cudaEventDestroy(start);
    cudaEventDestroy(done);
    return PMB_SUCCESS;
}
