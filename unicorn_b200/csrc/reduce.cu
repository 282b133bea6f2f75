// Element-wise reduction of subtasks' private output copies on the device:
// the built-in REDUCE_* callbacks of the reference (pmGetSubtaskReductionCallbackImpl,
// source/code/src/pmPublicDefinitions.cpp:749-800, and the loops of
// pmReducer::ReduceSubtasks, source/code/src/pmReducer.cpp:1073-1320), which
// the reference runs on the host over shadow memory.  Here the pm:: runtime
// keeps every subtask's copy in device memory and folds them with one launch
// per 128 sources:
//     dst[e] = src[0][e] (or dst[e] (+) src[0][e]) (+) src[1][e] (+) ...
// in source order (deterministic), each thread walking a grid-stride range of
// 16-byte vectors and every source read coalesced.  The pass reads nsrc +
// (init ? 0 : 1) arrays and writes one: HBM-bound.
#include "pmb_common.cuh"

namespace {

constexpr int kPerLaunch = 128;  // sources per launch, passed by value (1 KB of kernel parameters)

struct Sources {
    const void* p[kPerLaunch];
};

// Bitwise operations on FLOATS / DOUBLES act on the values converted to
// uint32 / uint64 (not on their bit patterns), as pmReducer.cpp:408-423 does.
template <typename T> struct BitwiseType { using type = T; };
template <> struct BitwiseType<float> { using type = uint32_t; };
template <> struct BitwiseType<double> { using type = uint64_t; };

// pmReducer::ReduceMemories (pmReducer.cpp:590-700): LOGICAL_XOR is value
// inequality (a != b), the logical ops yield 0 / 1.
template <typename T, int OP>
__device__ __forceinline__ T combine(T a, T b) {
    using B = typename BitwiseType<T>::type;
    if constexpr (OP == 0) return a + b;                                // ADD
    else if constexpr (OP == 1) return b < a ? b : a;                   // MIN (std::min)
    else if constexpr (OP == 2) return a < b ? b : a;                   // MAX (std::max)
    else if constexpr (OP == 3) return a * b;                           // PRODUCT
    else if constexpr (OP == 4) return (a != T(0) && b != T(0)) ? T(1) : T(0);  // LOGICAL_AND
    else if constexpr (OP == 5) return static_cast<T>(static_cast<B>(a) & static_cast<B>(b));  // BITWISE_AND
    else if constexpr (OP == 6) return (a != T(0) || b != T(0)) ? T(1) : T(0);  // LOGICAL_OR
    else if constexpr (OP == 7) return static_cast<T>(static_cast<B>(a) | static_cast<B>(b));  // BITWISE_OR
    else if constexpr (OP == 8) return a != b ? T(1) : T(0);            // LOGICAL_XOR
    else return static_cast<T>(static_cast<B>(a) ^ static_cast<B>(b));  // BITWISE_XOR
}

// 16-byte load of vector i of a source read once (evict-first streaming load).
template <typename Vec>
__device__ __forceinline__ Vec load_stream(const void* p, size_t i) {
    const uint4 u = __ldcs(static_cast<const uint4*>(p) + i);
    Vec v;
    static_assert(sizeof(Vec) == sizeof(uint4), "16-byte vectors");
    memcpy(&v, &u, sizeof(u));
    return v;
}

// Grid-stride over 16-byte vectors of elements when every pointer is 16-byte
// aligned (streaming loads: each source is read once), then the tail (or
// everything, for unaligned pointers) one element per thread.  The sources
// are folded in order for every element.
template <typename T, int OP>
__global__ void __launch_bounds__(256)
reduce_kernel(T* __restrict__ dst, const Sources srcs, int nsrc, size_t count, int init, int vec) {
    constexpr int V = 16 / sizeof(T);
    struct alignas(16) Vec {
        T v[V];
    };
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    const size_t tid = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const size_t nv = vec ? count / V : 0;
    for (size_t i = tid; i < nv; i += stride) {
        Vec a = load_stream<Vec>(srcs.p[0], i), b;
        if (!init) {
            b = reinterpret_cast<const Vec*>(dst)[i];
#pragma unroll
            for (int k = 0; k < V; ++k) a.v[k] = combine<T, OP>(b.v[k], a.v[k]);
        }
        for (int s = 1; s < nsrc; ++s) {
            b = load_stream<Vec>(srcs.p[s], i);
#pragma unroll
            for (int k = 0; k < V; ++k) a.v[k] = combine<T, OP>(a.v[k], b.v[k]);
        }
        reinterpret_cast<Vec*>(dst)[i] = a;
    }
    for (size_t e = nv * V + tid; e < count; e += stride) {
        const T first = static_cast<const T*>(srcs.p[0])[e];
        T acc = init ? first : combine<T, OP>(dst[e], first);
        for (int s = 1; s < nsrc; ++s) acc = combine<T, OP>(acc, static_cast<const T*>(srcs.p[s])[e]);
        dst[e] = acc;
    }
}

template <typename T, int OP>
int launch(void* dst, const void* const* srcs, int nsrc, size_t count, int init, cudaStream_t s) {
    bool vec = reinterpret_cast<uintptr_t>(dst) % 16 == 0;
    for (int i = 0; i < nsrc; ++i) vec = vec && reinterpret_cast<uintptr_t>(srcs[i]) % 16 == 0;
    const size_t per_block = 256 * (vec ? 16 / sizeof(T) : 1);
    const size_t blocks = (count + per_block - 1) / per_block;
    const unsigned grid = static_cast<unsigned>(blocks < 148 * 8 ? blocks : 148 * 8);
    for (int base = 0; base < nsrc; base += kPerLaunch) {
        Sources p{};
        const int n = nsrc - base < kPerLaunch ? nsrc - base : kPerLaunch;
        for (int i = 0; i < n; ++i) p.p[i] = srcs[base + i];
        reduce_kernel<T, OP><<<grid, 256, 0, s>>>(static_cast<T*>(dst), p, n, count, base == 0 ? init : 0, vec);
        PMB_CUDA_TRY(cudaGetLastError());
    }
    return PMB_SUCCESS;
}

template <typename T>
int dispatch_op(int op, void* dst, const void* const* srcs, int nsrc, size_t count, int init, cudaStream_t s) {
    switch (op) {
        case 0: return launch<T, 0>(dst, srcs, nsrc, count, init, s);
        case 1: return launch<T, 1>(dst, srcs, nsrc, count, init, s);
        case 2: return launch<T, 2>(dst, srcs, nsrc, count, init, s);
        case 3: return launch<T, 3>(dst, srcs, nsrc, count, init, s);
        case 4: return launch<T, 4>(dst, srcs, nsrc, count, init, s);
        case 5: return launch<T, 5>(dst, srcs, nsrc, count, init, s);
        case 6: return launch<T, 6>(dst, srcs, nsrc, count, init, s);
        case 7: return launch<T, 7>(dst, srcs, nsrc, count, init, s);
        case 8: return launch<T, 8>(dst, srcs, nsrc, count, init, s);
        case 9: return launch<T, 9>(dst, srcs, nsrc, count, init, s);
        default: return pmb::fail(PMB_INVALID_INDEX, "unknown reduction operation %d", op);
    }
}

}  // namespace

extern "C" size_t pmb_reduce_element_size(int type) {
    switch (type) {
        case 0: case 1: case 4: return 4;
        case 2: case 3: case 5: return 8;
        default: return 0;
    }
}

extern "C" int pmb_reduce_elementwise(int op, int type, void* d_dst, const void* const* srcs, int nsrc, size_t count,
                                      int init_from_first, void* stream) {
    PMB_CHECK_ARG(d_dst && srcs, "null pointer");
    PMB_CHECK_ARG(nsrc >= 1, "source count %d below 1", nsrc);
    const size_t es = pmb_reduce_element_size(type);
    if (es == 0) return pmb::fail(PMB_INVALID_INDEX, "unknown reduction data type %d", type);
    PMB_CHECK_ARG(reinterpret_cast<uintptr_t>(d_dst) % es == 0, "destination not aligned to its %zu-byte elements", es);
    for (int i = 0; i < nsrc; ++i)
        PMB_CHECK_ARG(srcs[i] && reinterpret_cast<uintptr_t>(srcs[i]) % es == 0,
                      "source %d null or not aligned to its %zu-byte elements", i, es);
    if (count == 0) return PMB_SUCCESS;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (type) {
        case 0: return dispatch_op<int32_t>(op, d_dst, srcs, nsrc, count, init_from_first, s);
        case 1: return dispatch_op<uint32_t>(op, d_dst, srcs, nsrc, count, init_from_first, s);
        case 2: return dispatch_op<int64_t>(op, d_dst, srcs, nsrc, count, init_from_first, s);
        case 3: return dispatch_op<uint64_t>(op, d_dst, srcs, nsrc, count, init_from_first, s);
        case 4: return dispatch_op<float>(op, d_dst, srcs, nsrc, count, init_from_first, s);
        default: return dispatch_op<double>(op, d_dst, srcs, nsrc, count, init_from_first, s);
    }
}
