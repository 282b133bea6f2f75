// pageRank subtask kernels: pull-style PageRank over CSR in-edges, plus the
// graph plumbing it needs on the device (R-MAT edge generator, CSR builder).
//
// Semantics (testSuite/pageRank/source/code/src/pageRank.cpp:237-276
// serialPageRank and :336-378 pageRank_cpu): one iteration computes
//     r'[v] = sum over edges u->v of  (d * r[u]) / outdeg(u)
// in fp32, with no teleport term ((1-d)/N is never added, :255-256); pages with
// no out-links contribute nothing.  The reference pushes each page's share to
// its targets with += (fp32 atomics on the GPU, pageRankCUDA.cu:46-65) and then
// reduces whole rank arrays across subtasks on the host (REDUCE_ADD).  Here
// every vertex PULLS over its in-edges, so each rank is owned by exactly one
// writer: no atomics, no cross-subtask reduction, and the result is
// deterministic run to run.
//
// Design.  The work is cut into slices of equal cost, one per warp: walking the
// vertices in order, every in-edge costs 1 and every vertex kVertexCost (its
// row bounds, segment bookkeeping and result), and each warp takes 2048 cost
// units (a merge-path split of row_ptr against the edge array).  So neither a
// high in-degree vertex (R-MAT concentrates edges on low ids) nor a long run
// of vertices without in-edges (R-MAT leaves most high ids empty; a fixed
// edge split once gave one warp 31k of them) can stall a warp.  A warp walks
// the edges of its slice 32 at a time: coalesced col[] loads, one
// gather of contrib[src] per edge, a segmented warp scan keyed by the owning
// vertex, and a shuffle that hands each segment total to the lane that owns
// the vertex.  A vertex whose in-edges cross slice boundaries leaves a partial
// sum in its owner slot and carries in later slices; a small fixup kernel adds
// them in slice order.  The per-source share contrib[u] = d*r[u]/outdeg(u) is
// produced in the epilogue of the previous iteration, so an iteration reads
// row_ptr, col, the gathered contrib values and outdeg, and writes one fp32
// per vertex.
#include "lookback.cuh"
#include "pmb_common.cuh"

extern "C" int pmb_radix_sort_pairs_u32(uint32_t* d_keys, uint32_t* d_alt, uint32_t* d_vals, uint32_t* d_vals_alt,
                                        size_t n, int begin_bit, int end_bit, int bits_per_pass, void* d_scratch,
                                        size_t scratch_bytes, void* stream);
extern "C" size_t pmb_radix_sort_scratch_bytes(size_t n, int bits_per_pass);
extern "C" size_t pmb_scan_scratch_bytes(size_t n);
extern "C" int pmb_inclusive_scan_u32_u64(const uint32_t* d_in, uint64_t* d_out, size_t n, void* d_scratch,
                                          size_t scratch_bytes, void* stream);

namespace {

constexpr int kSlice = 2048;      // cost units per warp
constexpr int kVertexCost = 16;   // cost of a vertex in units of one edge
constexpr int kWarpsPerCta = 8;
constexpr int kChunks = 4;      // 32-edge chunks whose loads are in flight together
constexpr int kCtaThreads = 32 * kWarpsPerCta;

// ---------------------------------------------------------------------------
// R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): each edge descends `scale`
// levels of the adjacency matrix, picking quadrant (src bit, dst bit) =
// (0,0), (0,1), (1,0), (1,1) with probabilities a, b, c, d.  Random bits come
// from SplitMix64 over (seed, edge index), so edge i is the same on any
// device and launch shape.
__device__ __forceinline__ uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void rmat_kernel(uint64_t seed, int scale, uint64_t n_edges, uint32_t ta, uint32_t tab, uint32_t tabc,
                            uint32_t* __restrict__ src, uint32_t* __restrict__ dst) {
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < n_edges;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t state = seed ^ (e * 0xD1B54A32D192ED03ull);
        uint32_t s = 0, d = 0;
        uint64_t bits = 0;
        for (int l = 0; l < scale; ++l) {
            if ((l & 1) == 0) bits = splitmix64(state);
            const uint32_t u = (l & 1) ? static_cast<uint32_t>(bits >> 32) : static_cast<uint32_t>(bits);
            const uint32_t sb = u >= tab ? 1u : 0u;                   // quadrants c, d
            const uint32_t db = (u >= ta && u < tab) || u >= tabc ? 1u : 0u;  // quadrants b, d
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        src[e] = s;
        dst[e] = d;
    }
}

// Out-degree histogram and sort keys (the destination).  An edge naming a
// vertex >= n_vertices gets key n_vertices, so it sorts past row_ptr[N] and is
// never traversed; it sets bit 2 of *err.
__global__ void degree_keys_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t n,
                                   uint32_t n_vertices, uint32_t* __restrict__ deg, uint32_t* __restrict__ keys,
                                   uint32_t* __restrict__ err) {
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < n;
         e += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = src[e], v = dst[e];
        if (u < n_vertices && v < n_vertices) {
            atomicAdd(&deg[u], 1u);
            keys[e] = v;
        } else {
            keys[e] = n_vertices;
            atomicOr(err, 2u);
        }
    }
}

// row_ptr[v] = first position of v in the sorted destination array.
__global__ void row_ptr_kernel(const uint32_t* __restrict__ sorted_dst, uint64_t n_edges, uint32_t n_vertices,
                               uint32_t* __restrict__ row_ptr) {
    const uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (v > n_vertices) return;
    uint64_t lo = 0, hi = n_edges;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (sorted_dst[mid] < v) lo = mid + 1; else hi = mid;
    }
    row_ptr[v] = static_cast<uint32_t>(lo);
}

// ---------------------------------------------------------------------------
// Plan.  // Cost position of vertex v's first item: C(v) = row_ptr[v] + kVertexCost * v.
// Vertex v occupies [C(v), C(v+1)): its in-edges, then kVertexCost units for
// its result.  Slice w covers cost [w*kSlice, (w+1)*kSlice).
//   e_start[w] : edges before the slice (its first edge; e_start[ns] = E);
//   own_lo[w]  : first vertex whose range starts in slice w or later -- the
//                slice owns (writes) the vertices [own_lo[w], own_lo[w+1]);
//   cont[w]    : the vertex that started before the slice and still has
//                in-edges in it (its sum there is carried), else -1.
__global__ void plan_kernel(const uint32_t* __restrict__ row_ptr, uint32_t n_vertices, uint64_t n_edges,
                            uint32_t n_slices, int32_t* __restrict__ own_lo, int32_t* __restrict__ cont,
                            uint32_t* __restrict__ e_start) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w > n_slices) return;
    if (w == n_slices) {
        own_lo[w] = static_cast<int32_t>(n_vertices);
        e_start[w] = static_cast<uint32_t>(n_edges);
        return;
    }
    const uint64_t pos = static_cast<uint64_t>(w) * kSlice;
    // va = last vertex with C(va) <= pos (C(0) = 0 <= pos)
    uint32_t lo = 0, hi = n_vertices - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        const uint64_t cm = static_cast<uint64_t>(row_ptr[mid]) + static_cast<uint64_t>(kVertexCost) * mid;
        if (cm <= pos) lo = mid; else hi = mid - 1;
    }
    const uint32_t va = lo;
    const uint64_t ca = static_cast<uint64_t>(row_ptr[va]) + static_cast<uint64_t>(kVertexCost) * va;
    const uint64_t indeg = row_ptr[va + 1] - row_ptr[va];
    const uint64_t into = pos - ca;  // cost units of va before the slice
    e_start[w] = static_cast<uint32_t>(row_ptr[va] + (into < indeg ? into : indeg));
    own_lo[w] = static_cast<int32_t>(into == 0 ? va : va + 1);
    cont[w] = (into > 0 && into < indeg) ? static_cast<int32_t>(va) : -1;
}

__global__ void init_contrib_kernel(const float* __restrict__ rank, const uint32_t* __restrict__ outdeg, float damping,
                                    uint32_t n, float* __restrict__ contrib) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint32_t od = outdeg[v];
    contrib[v] = od ? (damping * rank[v]) / static_cast<float>(od) : 0.0f;
}

__device__ __forceinline__ float finish(float r, uint32_t v, const uint32_t* __restrict__ outdeg, float damping,
                                        bool last) {
    if (last) return r;
    const uint32_t od = outdeg[v];
    return od ? (damping * r) / static_cast<float>(od) : 0.0f;
}

// The iteration kernels are chained by programmatic dependent launch: each
// waits here for the previous grid on the stream (at once when launched
// normally), then lets the next kernel's launch begin.
__device__ __forceinline__ void chain_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_dep(void (*kernel)(KArgs...), unsigned grid, unsigned threads, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// One iteration over all slices.  out[v] receives r'[v] (last iteration) or
// the next contrib d*r'[v]/outdeg(v); split vertices get their owner partial
// in out[v] and their later pieces in carry[slice].
__global__ void __launch_bounds__(kCtaThreads)
pull_kernel(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
            const uint32_t* __restrict__ outdeg, const float* __restrict__ contrib, const int32_t* __restrict__ own_lo,
            const int32_t* __restrict__ cont, const uint32_t* __restrict__ e_start, uint32_t n_slices,
            uint32_t n_vertices, float damping, int last, float* __restrict__ out, float* __restrict__ carry) {
    chain_wait();
    const uint32_t w = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (w >= n_slices) return;
    const int lane = threadIdx.x & 31;
    const uint64_t e_lo = e_start[w];
    const uint64_t e_hi = e_start[w + 1];
    const int32_t cv = cont[w];
    // Vertex list: [cv (if any), own_lo[w], ..., own_lo[w+1]-1]
    const int64_t first = cv >= 0 ? cv : own_lo[w];
    const int64_t end = own_lo[w + 1];
    for (int64_t vb = first; vb < end; vb += 32) {
        const int64_t v = vb + lane;
        const bool have = v < end;
        uint64_t s = 0, t = 0;
        if (have) {
            s = row_ptr[v];
            t = row_ptr[v + 1];
            if (s < e_lo) s = e_lo;
            if (t > e_hi) t = e_hi;
        }
        // Edge span of this group within the slice.
        const uint64_t g_lo = __shfl_sync(0xffffffffu, s, 0);
        const int64_t last_lane = (end - vb) < 32 ? (end - vb - 1) : 31;
        const uint64_t g_hi = __shfl_sync(0xffffffffu, t, static_cast<int>(last_lane));
        float acc = 0.0f;
        // kChunks 32-edge chunks per round: all their index loads, then all their
        // gathers, are issued before the first segmented scan, so each warp keeps
        // kChunks dependent load pairs in flight instead of one.
        for (uint64_t c0 = g_lo; c0 < g_hi; c0 += 32 * kChunks) {
            uint32_t u[kChunks];
            float vals[kChunks];
#pragma unroll
            for (int j = 0; j < kChunks; ++j) {
                const uint64_t e = c0 + 32 * j + lane;
                u[j] = e < g_hi ? __ldg(&col[e]) : n_vertices;
            }
#pragma unroll
            for (int j = 0; j < kChunks; ++j) vals[j] = u[j] < n_vertices ? __ldg(&contrib[u[j]]) : 0.0f;
#pragma unroll
            for (int j = 0; j < kChunks; ++j) {
                const uint64_t cb = c0 + 32 * j;
                if (cb >= g_hi) break;
                float val = vals[j];
                // Segment heads: first edge of every owner whose run starts in this chunk.
                const bool starts = have && s < t && s >= cb && s < cb + 32;
                uint32_t heads = __reduce_or_sync(0xffffffffu, starts ? (1u << (s - cb)) : 0u) | 1u;
                const int seg = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const float y = __shfl_up_sync(0xffffffffu, val, o);
                    if (lane - o >= seg) val += y;
                }
                // Owner lane pulls the total of its run's last edge in this chunk.
                const bool mine = have && s < t && s < cb + 32 && t > cb;
                const uint64_t last_e = (t < cb + 32 ? t : cb + 32) - 1;
                const int src_lane = mine ? static_cast<int>(last_e - cb) : lane;
                const float tot = __shfl_sync(0xffffffffu, val, src_lane);
                if (mine) acc += tot;
            }
        }
        if (have) {
            if (v == cv) {
                carry[w] = acc;
            } else {
                const bool split = row_ptr[v + 1] > e_hi;
                out[v] = split ? acc : finish(acc, static_cast<uint32_t>(v), outdeg, damping, last != 0);
            }
        }
    }
}

// Completes vertices whose in-edges span several slices: thread w handles the
// vertex whose first continuation slice is w, adding carries in slice order.
__global__ void fixup_kernel(const int32_t* __restrict__ cont, uint32_t n_slices, const uint32_t* __restrict__ outdeg,
                             float damping, int last, const float* __restrict__ carry, float* __restrict__ out) {
    chain_wait();
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_slices) return;
    const int32_t v = cont[w];
    if (v < 0 || (w > 0 && cont[w - 1] == v)) return;
    float r = out[v];
    for (uint32_t k = w; k < n_slices && cont[k] == v; ++k) r += carry[k];
    out[v] = finish(r, static_cast<uint32_t>(v), outdeg, damping, last != 0);
}

// ---------------------------------------------------------------------------
// The reference's web-dump pages (pageRank.cpp:53-111): per page a u32
// out-link count followed by max_outlinks u32 slots, the first `count` of
// them 1-based target ids; pages are `stride` = max_outlinks + 1 words apart.

// counts[p] = the page's out-link count (clamped to the slots; bit 3 of *err
// when a count exceeds them).
__global__ void webdump_counts_kernel(const uint32_t* __restrict__ dump, uint32_t n_pages, uint32_t stride,
                                      uint32_t* __restrict__ counts, uint32_t* __restrict__ err) {
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < n_pages;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t c = dump[p * stride];
        if (c > stride - 1) {
            c = stride - 1;
            atomicOr(err, 4u);
        }
        counts[p] = c;
    }
}

// Edge list in page order: page p's edges at [incl[p] - counts[p], incl[p]),
// (source p, 0-based target).  Targets outside [1, n_vertices] become
// n_vertices, which the CSR builder drops (and flags); positions at or past
// n_edges are skipped and set bit 4 of *err.  Eight lanes per page.
__global__ void webdump_edges_kernel(const uint32_t* __restrict__ dump, uint32_t n_pages, uint32_t stride,
                                     const uint32_t* __restrict__ counts, const uint64_t* __restrict__ incl,
                                     uint32_t n_vertices, uint64_t n_edges, uint32_t* __restrict__ src,
                                     uint32_t* __restrict__ dst, uint32_t* __restrict__ err) {
    const uint64_t groups = static_cast<uint64_t>(gridDim.x) * blockDim.x / 8;
    const uint32_t l8 = threadIdx.x & 7;
    for (uint64_t p = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / 8; p < n_pages; p += groups) {
        const uint32_t c = counts[p];
        const uint64_t base = incl[p] - c;
        const uint32_t* row = dump + p * stride + 1;
        for (uint32_t k = l8; k < c; k += 8) {
            const uint64_t e = base + k;
            if (e >= n_edges) {
                atomicOr(err, 8u);
                continue;
            }
            const uint32_t t = row[k];
            src[e] = static_cast<uint32_t>(p);
            dst[e] = (t >= 1 && t <= n_vertices) ? t - 1 : n_vertices;
        }
    }
}

__global__ void or_word_kernel(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src) { *dst |= *src; }

// One step of the reference's push (pageRankCUDA.cu:46-65, pageRank_cpu
// :336-378): every page adds (d * r) / count to each target.  Eight lanes per
// page read its slots coalesced; the adds are fire-and-forget fp32 reductions
// in L2 (the order of the adds is not fixed, as with the reference's atomics).
__global__ void webdump_push_kernel(const uint32_t* __restrict__ dump, uint32_t n_pages, uint32_t stride,
                                    const float* __restrict__ rank_in, float init, float damping,
                                    float* __restrict__ out, uint32_t n_vertices, uint32_t* __restrict__ err) {
    const uint64_t groups = static_cast<uint64_t>(gridDim.x) * blockDim.x / 8;
    const uint32_t l8 = threadIdx.x & 7;
    bool bad = false;
    for (uint64_t p = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / 8; p < n_pages; p += groups) {
        const uint32_t* row = dump + p * stride;
        uint32_t c = row[0];
        if (c > stride - 1) {
            c = stride - 1;
            bad = true;
        }
        if (c == 0) continue;
        const float r = rank_in ? rank_in[p] : init;
        const float incr = (damping * r) / static_cast<float>(c);
        for (uint32_t k = l8; k < c; k += 8) {
            const uint32_t t = row[1 + k];
            if (t >= 1 && t <= n_vertices) atomicAdd(&out[t - 1], incr);
            else bad = true;
        }
    }
    if (bad && err) atomicOr(err, 2u);
}

uint32_t slices_for(uint32_t n_vertices, uint64_t n_edges) {
    const uint64_t cost = n_edges + static_cast<uint64_t>(kVertexCost) * n_vertices;
    return static_cast<uint32_t>((cost + kSlice - 1) / kSlice);
}

unsigned grid_for(uint64_t n, int threads, unsigned cap) {
    const uint64_t g = (n + threads - 1) / threads;
    return static_cast<unsigned>(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

extern "C" int pmb_rmat_edges(uint64_t seed, int scale, uint64_t n_edges, double a, double b, double c,
                              uint32_t* d_src, uint32_t* d_dst, void* stream) {
    PMB_CHECK_ARG(d_src && d_dst, "null pointer");
    PMB_CHECK_ARG(scale >= 1 && scale <= 32, "scale %d outside [1,32]", scale);
    PMB_CHECK_ARG(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, "bad R-MAT probabilities");
    if (n_edges == 0) return PMB_SUCCESS;
    const double two32 = 4294967296.0;
    auto thr = [&](double p) -> uint32_t { const double x = p * two32; return x >= two32 ? 0xffffffffu : static_cast<uint32_t>(x); };
    rmat_kernel<<<grid_for(n_edges, 256, 148 * 64), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        seed, scale, n_edges, thr(a), thr(a + b), thr(a + b + c), d_src, d_dst);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

extern "C" size_t pmb_csr_scratch_bytes(uint32_t n_vertices, uint64_t n_edges) {
    (void)n_vertices;
    // two edge-sized temporaries (sorted keys / values ping-pong) + sort scratch
    const size_t e4 = (static_cast<size_t>(n_edges) * 4 + 255) & ~static_cast<size_t>(255);
    return 256 + 3 * e4 + pmb_radix_sort_scratch_bytes(n_edges, 8);
}

extern "C" int pmb_csr_by_destination(const uint32_t* d_src, const uint32_t* d_dst, uint32_t n_vertices,
                                      uint64_t n_edges, uint32_t* d_row_ptr, uint32_t* d_col, uint32_t* d_out_degree,
                                      void* d_scratch, size_t scratch_bytes, void* stream) {
    PMB_CHECK_ARG(d_src && d_dst && d_row_ptr && d_col && d_out_degree && d_scratch, "null pointer");
    PMB_CHECK_ARG(n_vertices >= 1, "graph without vertices");
    PMB_CHECK_ARG(n_edges < (1ull << 30), "edge count above 2^30");
    PMB_CHECK_ARG(scratch_bytes >= pmb_csr_scratch_bytes(n_vertices, n_edges), "CSR scratch too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t e4 = (static_cast<size_t>(n_edges) * 4 + 255) & ~static_cast<size_t>(255);
    uint32_t* hdr = static_cast<uint32_t*>(d_scratch);  // hdr[1]: error word
    char* base = static_cast<char*>(d_scratch) + 256;
    uint32_t* keys = reinterpret_cast<uint32_t*>(base);
    uint32_t* keys_alt = reinterpret_cast<uint32_t*>(base + e4);
    uint32_t* vals_alt = reinterpret_cast<uint32_t*>(base + 2 * e4);
    void* sort_scratch = base + 3 * e4;
    PMB_CUDA_TRY(cudaMemsetAsync(d_out_degree, 0, 4ull * n_vertices, s));
    PMB_CUDA_TRY(cudaMemsetAsync(hdr, 0, 256, s));
    if (n_edges) {
        degree_keys_kernel<<<grid_for(n_edges, 256, 148 * 32), 256, 0, s>>>(d_src, d_dst, n_edges, n_vertices,
                                                                             d_out_degree, keys, &hdr[1]);
        PMB_CUDA_TRY(cudaGetLastError());
        PMB_CUDA_TRY(cudaMemcpyAsync(d_col, d_src, 4 * n_edges, cudaMemcpyDeviceToDevice, s));
        int bits_end = 8;  // keys go up to n_vertices inclusive
        while (bits_end < 32 && (static_cast<uint64_t>(n_vertices) >> bits_end)) bits_end += 8;
        const int st = pmb_radix_sort_pairs_u32(keys, keys_alt, d_col, vals_alt, n_edges, 0, bits_end, 8,
                                                sort_scratch, pmb_radix_sort_scratch_bytes(n_edges, 8), stream);
        if (st != PMB_SUCCESS) return st;
    }
    row_ptr_kernel<<<grid_for(static_cast<uint64_t>(n_vertices) + 1, 256, 0x7fffffffu), 256, 0, s>>>(
        keys, n_edges, n_vertices, d_row_ptr);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

extern "C" size_t pmb_pagerank_plan_bytes(uint32_t n_vertices, uint64_t n_edges) {
    return 12ull * (slices_for(n_vertices, n_edges) + 1);
}

extern "C" int pmb_pagerank_plan(const uint32_t* d_row_ptr, uint32_t n_vertices, uint64_t n_edges, void* d_plan,
                                 size_t plan_bytes, void* stream) {
    PMB_CHECK_ARG(d_row_ptr && d_plan, "null pointer");
    PMB_CHECK_ARG(plan_bytes >= pmb_pagerank_plan_bytes(n_vertices, n_edges), "plan buffer too small");
    PMB_CHECK_ARG(n_vertices >= 1, "no vertices");
    const uint32_t ns = slices_for(n_vertices, n_edges);
    int32_t* own_lo = static_cast<int32_t*>(d_plan);
    int32_t* cont = own_lo + ns + 1;
    uint32_t* e_start = reinterpret_cast<uint32_t*>(cont + ns + 1);
    plan_kernel<<<grid_for(ns + 1ull, 256, 0x7fffffffu), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d_row_ptr, n_vertices, n_edges, ns, own_lo, cont, e_start);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

extern "C" size_t pmb_pagerank_work_bytes(uint32_t n_vertices, uint64_t n_edges) {
    return 8ull * n_vertices + 4ull * slices_for(n_vertices, n_edges) + 256;
}

extern "C" int pmb_pagerank(const uint32_t* d_row_ptr, const uint32_t* d_col, const uint32_t* d_out_degree,
                            uint32_t n_vertices, uint64_t n_edges, const void* d_plan, float damping, int iterations,
                            const float* d_rank_in, float* d_rank_out, void* d_work, size_t work_bytes, void* stream) {
    PMB_CHECK_ARG(d_row_ptr && d_col && d_out_degree && d_plan && d_rank_in && d_rank_out && d_work, "null pointer");
    PMB_CHECK_ARG(iterations >= 0, "negative iteration count");
    PMB_CHECK_ARG(n_vertices >= 1 && n_edges < (1ull << 32), "bad graph size");
    PMB_CHECK_ARG(work_bytes >= pmb_pagerank_work_bytes(n_vertices, n_edges), "work buffer too small");
    PMB_CHECK_ARG(d_rank_in != d_rank_out, "rank input and output must differ");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (iterations == 0) {
        PMB_CUDA_TRY(cudaMemcpyAsync(d_rank_out, d_rank_in, 4ull * n_vertices, cudaMemcpyDeviceToDevice, s));
        return PMB_SUCCESS;
    }
    const uint32_t ns = slices_for(n_vertices, n_edges);
    const int32_t* own_lo = static_cast<const int32_t*>(d_plan);
    const int32_t* cont = own_lo + ns + 1;
    const uint32_t* e_start = reinterpret_cast<const uint32_t*>(cont + ns + 1);
    float* ca = static_cast<float*>(d_work);
    float* cbuf = ca + n_vertices;
    float* carry = cbuf + n_vertices;
    init_contrib_kernel<<<grid_for(n_vertices, 256, 0x7fffffffu), 256, 0, s>>>(d_rank_in, d_out_degree, damping,
                                                                              n_vertices, ca);
    PMB_CUDA_TRY(cudaGetLastError());
    const unsigned pgrid = (ns + kWarpsPerCta - 1) / kWarpsPerCta;
    for (int it = 0; it < iterations; ++it) {
        const int last = it == iterations - 1;
        float* dst = last ? d_rank_out : cbuf;
        if (ns == 0) {
            PMB_CUDA_TRY(cudaMemsetAsync(dst, 0, 4ull * n_vertices, s));
        } else {
            PMB_CUDA_TRY(launch_dep(pull_kernel, pgrid, kCtaThreads, s, d_row_ptr, d_col, d_out_degree,
                                    static_cast<const float*>(ca), own_lo, cont, e_start, ns, n_vertices, damping, last,
                                    dst, carry));
            PMB_CUDA_TRY(launch_dep(fixup_kernel, grid_for(ns, 256, 0x7fffffffu), 256, s, cont, ns, d_out_degree,
                                    damping, last, static_cast<const float*>(carry), dst));
        }
        float* t = ca;
        ca = cbuf;
        cbuf = t;
    }
    return PMB_SUCCESS;
}

// ---------------------------------------------------------------------------
// Web-dump pages -> CSR by destination, and the reference's push step.

namespace {
size_t align256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }
}  // namespace

extern "C" size_t pmb_webdump_csr_scratch_bytes(uint32_t n_pages, uint32_t n_vertices, uint64_t n_edges) {
    // CSR builder scratch (its header first) | counts | inclusive offsets | scan scratch | src | dst
    return align256(pmb_csr_scratch_bytes(n_vertices, n_edges)) + align256(4ull * n_pages) +
           align256(8ull * n_pages) + align256(pmb_scan_scratch_bytes(n_pages)) + 2 * align256(4ull * n_edges) + 256;
}

extern "C" int pmb_csr_from_webdump(const uint32_t* d_dump, uint32_t n_pages, uint32_t max_outlinks,
                                    uint32_t n_vertices, uint64_t n_edges, uint32_t* d_row_ptr, uint32_t* d_col,
                                    uint32_t* d_out_degree, void* d_scratch, size_t scratch_bytes, void* stream) {
    PMB_CHECK_ARG(d_dump && d_row_ptr && d_col && d_out_degree && d_scratch, "null pointer");
    PMB_CHECK_ARG(n_pages >= 1 && n_pages <= n_vertices, "pages %u outside [1, n_vertices = %u]", n_pages, n_vertices);
    PMB_CHECK_ARG(max_outlinks >= 1 && max_outlinks < 0xffffffffu, "bad max_outlinks %u", max_outlinks);
    PMB_CHECK_ARG(n_edges < (1ull << 30), "edge count above 2^30");
    PMB_CHECK_ARG(scratch_bytes >= pmb_webdump_csr_scratch_bytes(n_pages, n_vertices, n_edges), "scratch too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* p = static_cast<char*>(d_scratch);
    const size_t csr_bytes = align256(pmb_csr_scratch_bytes(n_vertices, n_edges));
    uint32_t* hdr = static_cast<uint32_t*>(d_scratch);
    char* q = p + csr_bytes;
    uint32_t* own_err = reinterpret_cast<uint32_t*>(q);
    q += 256;
    uint32_t* counts = reinterpret_cast<uint32_t*>(q);
    q += align256(4ull * n_pages);
    uint64_t* incl = reinterpret_cast<uint64_t*>(q);
    q += align256(8ull * n_pages);
    void* scan_scratch = q;
    const size_t scan_bytes = align256(pmb_scan_scratch_bytes(n_pages));
    q += scan_bytes;
    uint32_t* src = reinterpret_cast<uint32_t*>(q);
    q += align256(4ull * n_edges);
    uint32_t* dst = reinterpret_cast<uint32_t*>(q);
    const uint32_t stride = max_outlinks + 1;
    PMB_CUDA_TRY(cudaMemsetAsync(own_err, 0, 4, s));
    if (n_edges) PMB_CUDA_TRY(cudaMemsetAsync(dst, 0xff, 4ull * n_edges, s));  // unfilled slots are dropped
    webdump_counts_kernel<<<grid_for(n_pages, 256, 148 * 32), 256, 0, s>>>(d_dump, n_pages, stride, counts, own_err);
    PMB_CUDA_TRY(cudaGetLastError());
    int st = pmb_inclusive_scan_u32_u64(counts, incl, n_pages, scan_scratch, scan_bytes, stream);
    if (st != PMB_SUCCESS) return st;
    webdump_edges_kernel<<<grid_for(8ull * n_pages, 256, 148 * 32), 256, 0, s>>>(
        d_dump, n_pages, stride, counts, incl, n_vertices, n_edges, src, dst, own_err);
    PMB_CUDA_TRY(cudaGetLastError());
    st = pmb_csr_by_destination(src, dst, n_vertices, n_edges, d_row_ptr, d_col, d_out_degree, d_scratch,
                                csr_bytes, stream);
    if (st != PMB_SUCCESS) return st;
    or_word_kernel<<<1, 1, 0, s>>>(&hdr[1], own_err);  // the builder cleared its header: fold ours in
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}

extern "C" int pmb_webdump_push(const uint32_t* d_dump, uint32_t n_pages, uint32_t max_outlinks,
                                const float* d_rank_in, float initial_rank, float damping, float* d_out,
                                uint32_t n_vertices, uint32_t* d_err, void* stream) {
    PMB_CHECK_ARG(d_dump && d_out, "null pointer");
    PMB_CHECK_ARG(n_vertices >= 1, "no vertices");
    PMB_CHECK_ARG(max_outlinks >= 1 && max_outlinks < 0xffffffffu, "bad max_outlinks %u", max_outlinks);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    PMB_CUDA_TRY(cudaMemsetAsync(d_out, 0, 4ull * n_vertices, s));
    if (n_pages == 0) return PMB_SUCCESS;
    webdump_push_kernel<<<grid_for(8ull * n_pages, 256, 148 * 16), 256, 0, s>>>(
        d_dump, n_pages, max_outlinks + 1, d_rank_in, initial_rank, damping, d_out, n_vertices, d_err);
    PMB_CUDA_TRY(cudaGetLastError());
    return PMB_SUCCESS;
}
