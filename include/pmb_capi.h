/*
 * pmb_capi.h -- C ABI of the B200 subtask execution path (libpmb.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status whose values are the pmStatus codes of the pm:: API
 * (pmPublicDefinitions.h), and never throws.  Device pointers are CUDA device
 * addresses on the current device; `stream` is a cudaStream_t passed as void*
 * (NULL = legacy default stream).  Host pointers are plain host memory (pinned
 * memory is faster but not required).
 *
 * Each declaration names the reference interface it replaces
 * (iitd-plos/unicorn, paths relative to that project).
 */
#ifndef PMB_CAPI_H
#define PMB_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: identical numbering to pm::pmStatus. */
enum {
    PMB_SUCCESS = 0,                  /* pmSuccess */
    PMB_STATUS_UNAVAILABLE = 2,       /* pmStatusUnavailable */
    PMB_FATAL_ERROR = 3,              /* pmFatalError */
    PMB_INVALID_INDEX = 7,            /* pmInvalidIndex: bad argument */
    PMB_MEMORY_ERROR = 11,            /* pmMemoryError: allocation failed */
    PMB_GRAPHICS_CARD_ERROR = 14,     /* pmGraphicsCardError: CUDA error */
    PMB_BEYOND_LIMITS = 15,           /* pmBeyondComputationalLimits: size too large */
    PMB_DATA_PROCESSING_FAILURE = 19, /* pmDataProcessingFailure: device-side check failed */
    PMB_NO_COMPATIBLE_DEVICE = 20     /* pmNoCompatibleDevice: no sm_100 GPU */
};

/* Last error message of the calling thread (empty string if none). */
const char* pmb_last_error(void);

/* Library version "major_minor_update" (replaces pm::pmGetLibVersion,
 * source/code/src/pmPublicDefinitions.cpp). */
const char* pmb_version(void);

/* 1 if device `dev` is an sm_100 part this library was built for, else 0. */
int pmb_device_supported(int dev);

/* ------------------------------------------------------------------------ */
/* Device layer: what the pm:: runtime (libpmlib.so) uses instead of calling  */
/* the CUDA runtime itself (replaces pmCudaInterface's dlsym'd calls,        */
/* source/code/src/pmCudaInterface.cu:69-173, :336-339, :474-550).           */
/* ------------------------------------------------------------------------ */

/* Copy directions for pmb_memcpy_async / pmb_memcpy2d_async. */
#define PMB_H2D 0
#define PMB_D2H 1
#define PMB_D2D 2
#define PMB_COPY_DEFAULT 3

int pmb_device_count(int* count);
int pmb_set_device(int dev);
int pmb_device_properties(int dev, char* name, size_t name_len, int* sm_count, int* cc_major, int* cc_minor);
int pmb_mem_get_info(size_t* free_bytes, size_t* total_bytes);
int pmb_malloc(void** p, size_t bytes);
int pmb_free(void* p);
int pmb_malloc_async(void** p, size_t bytes, void* stream);
int pmb_free_async(void* p, void* stream);
int pmb_host_alloc(void** p, size_t bytes); /* pinned, portable */
int pmb_host_free(void* p);
int pmb_stream_create(void** stream);        /* non-blocking stream */
int pmb_stream_destroy(void* stream);
int pmb_stream_synchronize(void* stream);
int pmb_event_create(void** event, int timing);
int pmb_event_destroy(void* event);
int pmb_event_record(void* event, void* stream);
int pmb_event_query(void* event);            /* PMB_SUCCESS done, PMB_STATUS_UNAVAILABLE pending */
int pmb_event_synchronize(void* event);
int pmb_event_elapsed_ms(void* start, void* end, float* ms);
int pmb_stream_wait_event(void* stream, void* event);
int pmb_memcpy_async(void* dst, const void* src, size_t bytes, int kind, void* stream);
int pmb_memcpy2d_async(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                       int kind, void* stream);
int pmb_memset_async(void* p, int value, size_t bytes, void* stream);
/* Copy n_ranges byte ranges d_src + src -> d_dst + dst in one launch on
 * `stream`; d_ranges is a device array.  Ranges must not overlap their
 * destinations.  Replaces the range-by-range copies of ordered
 * redistribution (source/code/src/pmRedistributor.cpp:240-283). */
typedef struct pmb_copy_range {
    uint64_t src, dst, len;
} pmb_copy_range;
int pmb_copy_ranges(void* d_dst, const void* d_src, const pmb_copy_range* d_ranges, int n_ranges, void* stream);
/* cudaLaunchKernel of a __global__ function pointer (an app's
 * subtask_gpu_cuda kernel) with the argument array `args`. */
int pmb_launch_kernel(const void* fn, unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by, unsigned bz,
                      unsigned smem, void** args, void* stream);
int pmb_device_synchronize(void);
/* Keep blocks freed with pmb_free_async in the device's default pool for
 * reuse (release threshold = unlimited). */
int pmb_mempool_retain(int dev);
/* Map device memory into the default pool now, until it holds `bytes` (less
 * if the device cannot provide them); *reserved (may be null) gets the pool's
 * size.  Growing the pool later, while kernels and copies are in flight,
 * stalls them: the pm:: runtime reserves its device budget at pmInitialize,
 * as the reference's CUDA stub reserves its chunk collections up front
 * (source/code/src/pmExecutionStub.cpp:3616-3640 pmStubCUDA::ReserveMemory,
 * chunks from pmDataTypes.cpp:505-509). */
int pmb_mempool_reserve(int dev, size_t bytes, size_t* reserved);
/* Return idle pool memory beyond keep_bytes to the device. */
int pmb_mempool_trim(int dev, size_t keep_bytes);
/* Free device memory plus memory the default pool holds but does not use. */
int pmb_mem_available(int dev, size_t* available);
/* Stream capture into an instantiated CUDA graph, and its launch. */
int pmb_graph_begin_capture(void* stream);
int pmb_graph_end_capture(void* stream, void** graph_exec);
int pmb_graph_launch(void* graph_exec, void* stream);
int pmb_graph_destroy(void* graph_exec);

/* ------------------------------------------------------------------------ */
/* imageFiltering: 2-D (2r+1)^2 RGB stencil                                  */
/* ------------------------------------------------------------------------ */

/* Maximum filter geometry, as in testSuite/imageFiltering/.../imageFiltering.h:58-61. */
#define PMB_IMGF_MAX_FILTER_DIM 32
#define PMB_IMGF_MAX_RADIUS 15

/* Accumulation mode.
 *  WRAP : reference semantics -- products summed into a signed char, i.e. the
 *         output byte is (sum of in*f) mod 256 (imageFiltering.cpp:428-467).
 *  CLAMP: inputs as unsigned bytes, exact int sum, output clamped to [0,255]. */
#define PMB_IMGF_WRAP 0
#define PMB_IMGF_CLAMP 1

/* One subtask (output rectangle) of an image-filter task.  The input view is
 * the address space as the reference lays it out: rows stored bottom-up
 * (buffer row b holds image row H-1-b), 3 bytes per pixel.  `in` points at
 * buffer row `in_row0`, pixel column `in_col0` of that layout (NATURAL view:
 * in_row0 = in_col0 = 0 and in_pitch = 3W; COMPACT view: the first subscribed
 * row/col).  The output view is top-down: `out` points at image row
 * `out_row0`, column `out_col0`.  The subtask writes image rows [r0,r1) x
 * columns [c0,c1); every input pixel read lies in image rows
 * [max(0,r0-R), min(H-1,r1-1+R)] and columns [max(0,c0-R), min(W-1,c1-1+R)],
 * which is exactly the reference's input subscription
 * (imageFiltering.cpp:353-361). */
typedef struct pmb_imgf_item {
    const uint8_t* in;
    uint8_t* out;
    int64_t in_pitch;   /* bytes between consecutive buffer rows of `in` */
    int64_t out_pitch;  /* bytes between consecutive image rows of `out` */
    int32_t width, height;      /* full image W, H in pixels */
    int32_t in_row0, in_col0;   /* buffer row / pixel column `in` points at */
    int32_t out_row0, out_col0; /* image row / pixel column `out` points at */
    int32_t r0, r1, c0, c1;     /* output rectangle (image coordinates) */
} pmb_imgf_item;

/* Filter every item of `items` (host array of n_items entries, 1 <= n_items
 * <= PMB_IMGF_MAX_ITEMS; item pointers are device pointers) with one
 * (2*radius+1)^2 filter in ONE launch on `stream`.  `filter` is a host
 * PMB_IMGF_MAX_FILTER_DIM x PMB_IMGF_MAX_FILTER_DIM row-major signed-byte
 * array indexed [ky][kx] (the layout of imageFilterTaskConf::filter,
 * imageFiltering.h:96-109).  Replaces imageFilter_cudaLaunchFunc /
 * imageFilter_cuda (testSuite/imageFiltering/source/code/src/
 * imageFilteringCUDA.cu:295-342, :86-231) for a batch of subtasks; the result
 * per subtask equals imageFilter_cpu (imageFiltering.cpp:379-472).  The item
 * table travels in the kernel's parameter block, so the call allocates
 * nothing and the host array may be reused as soon as the call returns. */
#define PMB_IMGF_MAX_ITEMS 256
int pmb_image_filter(const pmb_imgf_item* items, int n_items,
                     const int8_t* filter, int radius, int mode, void* stream);

/* The rectangles one pmb_image_filter call filters for `items` (host only,
 * no device work): items whose views are whole-row layouts (in_pitch =
 * out_pitch = 3W) of the same input and output images and whose output
 * rectangles are adjacent -- same rows with touching columns, or same columns
 * with touching rows -- are merged into one item covering both; empty
 * rectangles are dropped; other items are kept as they are.  Writes at most
 * n_items items to `out` and their count to `*n_out`.  No counterpart in the
 * reference. */
int pmb_image_filter_cover(const pmb_imgf_item* items, int n_items, pmb_imgf_item* out, int* n_out);

/* Error word of the stencil kernels on the current device (synchronous copy;
 * `clear` resets it): 0 = clean; 1 = a bounded wait of a tensor-core stencil
 * launch (tile staging or its matrix products) expired, and that launch's
 * output is not valid.  No counterpart in the reference. */
int pmb_image_filter_error(int clear, uint32_t* error_out);

/* Whole-image convenience form: one item covering the full image with
 * NATURAL views (in_pitch = out_pitch = 3W). */
int pmb_image_filter_full(const uint8_t* d_in, uint8_t* d_out, int width, int height,
                          const int8_t* filter, int radius, int mode, void* stream);

/* Host-to-host form: h_in / h_out are host images (pinned memory overlaps the
 * copies), d_in / d_out device buffers of the same size (3*W*H bytes).  The
 * image is processed in `bands` row bands (1..256) pipelined over three
 * streams: band k+1 uploads while band k is filtered and band k-1 downloads.
 * `stream` is the caller's stream; the call's work is complete when work
 * enqueued on `stream` after it starts.  Replaces the staging of
 * pmStubCUDA (source/code/src/pmExecutionStub.cpp:3655-3847) for a whole
 * imageFiltering task whose address spaces live in host memory. */
int pmb_image_filter_host(const uint8_t* h_in, uint8_t* h_out, uint8_t* d_in, uint8_t* d_out, int width, int height,
                          const int8_t* filter, int radius, int mode, int bands, void* stream);

/* Plain GPU form: one thread per output pixel, 3*(2r+1)^2 byte loads from
 * global memory and scalar multiply-adds; NATURAL views only.  The
 * one-task-at-a-time baseline the stencil kernel is compared with. */
int pmb_image_filter_plain(const uint8_t* d_in, uint8_t* d_out, int width, int height,
                           const int8_t* filter, int radius, int mode, void* stream);

/* ------------------------------------------------------------------------ */
/* Subtask reduction (REDUCE_* built-ins)                                   */
/* ------------------------------------------------------------------------ */

/* Bytes per element of a pmReductionDataType (INTS, UNSIGNED_INTS, LONGS,
 * UNSIGNED_LONGS, FLOATS, DOUBLES = 0..5); 0 for an unknown type. */
size_t pmb_reduce_element_size(int type);

/* Element-wise fold of nsrc device arrays of `count` elements into d_dst, in
 * source order: d_dst[e] = src0[e] (init_from_first) or d_dst[e] op src0[e],
 * then op src1[e], ... .  op and type take the pmReductionOpType /
 * pmReductionDataType values (bitwise ops on FLOATS / DOUBLES act on the
 * values converted to uint32 / uint64, LOGICAL_XOR is a != b, as the
 * reference's reducer defines them); `srcs` is a
 * HOST array of nsrc device pointers (passed to the kernels by value, 128 per
 * launch).  Every pointer must be aligned to the element size
 * (PMB_INVALID_INDEX otherwise).  Launches on `stream`, no synchronisation.
 * Replaces the host loops of the built-in reduction callbacks
 * (source/code/src/pmReducer.cpp:1073-1320, pmPublicDefinitions.cpp:749-800)
 * for subtask copies the pm:: runtime keeps in device memory. */
int pmb_reduce_elementwise(int op, int type, void* d_dst, const void* const* d_srcs, int nsrc, size_t count,
                           int init_from_first, void* stream);

/* Sentinel compression of a reduction output (zero is the sentinel) for its
 * copy to the host, in the reference's compressed form: a uint32 count, the
 * count non-zero elements, then their count uint32 indices, index order;
 * compressed only when count < 0.4 x elements
 * (source/code/src/pmCudaInterface.cu:380-472 CompressForSentinel,
 * pmExecutionStub.cpp:3850-3950, pmInternalDefinitions.h:223-224).  `type` is
 * a pmReductionDataType (INTS .. DOUBLES = 0..5); elements are stored as
 * 32-bit words.  pmb_sentinel_compress writes the count word always and the
 * rest only when the data compresses (three launches on `stream`, no
 * synchronisation); read the count, then pmb_sentinel_compressed tells
 * whether to copy 4 + count x (element size + 4) bytes or the data as it is.
 * d_dst needs pmb_sentinel_capacity_bytes, d_scratch (16-byte aligned)
 * pmb_sentinel_scratch_bytes.  pmb_sentinel_expand restores a host array
 * (UncompressSentinelCompressedData, pmExecutionStub.cpp:3878-3950). */
size_t pmb_sentinel_capacity_bytes(int type, size_t length);
size_t pmb_sentinel_scratch_bytes(int type, size_t length);
int pmb_sentinel_compress(int type, const void* d_src, size_t length, void* d_dst, size_t capacity, void* d_scratch,
                          size_t scratch_bytes, void* stream);
int pmb_sentinel_compressed(int type, size_t length, uint32_t count);
int pmb_sentinel_expand(int type, const void* h_src, void* h_dst, size_t length);

/* ------------------------------------------------------------------------ */
/* prefixSum: inclusive scan                                                */
/* ------------------------------------------------------------------------ */

/* Bytes of device scratch pmb_inclusive_scan_u32_u64 needs for n elements
 * (a 256-byte header and one 64-bit status word per 16384-element tile). */
size_t pmb_scan_scratch_bytes(size_t n);

/* out[i] = in[0] + ... + in[i] with 64-bit sums, n <= 2^30: one memset of the
 * scratch and one single-pass launch on `stream` (decoupled look-back over
 * 16384-element tiles; every look-back wait is bounded and reported in the
 * scratch error word).  d_in, d_out and d_scratch are device pointers,
 * 16-byte aligned.  Replaces prefixSum_cudaLaunchFunc / prefixSum_cuda /
 * elemAdd_cuda and the host scan of subtask totals
 * (testSuite/prefixSum/source/code/src/prefixSumCUDA.cu:68-267,
 * prefixSum.cpp:189-294); result equals serialPrefixSum (prefixSum.cpp:47-53)
 * widened to uint64. */
int pmb_inclusive_scan_u32_u64(const uint32_t* d_in, uint64_t* d_out, size_t n, void* d_scratch,
                               size_t scratch_bytes, void* stream);

/* Allocation-free form of pmb_inclusive_scan_u32_u64, with no counterpart in
 * the reference.  It is for callers that must not allocate device memory: a
 * pm:: subtask_gpu_custom callback may only enqueue work on the stream it is
 * handed (cudaMalloc/cudaFree synchronise the device and would stall every
 * subtask in flight), and a service that fixes its memory budget up front
 * cannot let a library grow it.  The scan's scratch (tile counter, error word
 * and tile status words) is a fixed 1 MiB device array inside libpmb.so, held
 * by every GPU that loads the library until the process exits; the call
 * allocates nothing, and n is limited to PMB_SCAN_NOALLOC_MAX_ELEMS (longer
 * inputs return PMB_BEYOND_LIMITS).  The first call on a device looks up the
 * array's device address with that device current and keeps it for the life
 * of the process: make that first call before any stream capture, and do not
 * use the entry point after cudaDeviceReset.  All calls share the one array
 * (each clears it on its stream before use), so calls whose work overlaps on
 * the GPU -- on different streams, or from different threads -- race and
 * must be serialised by the caller. */
#define PMB_SCAN_NOALLOC_MAX_ELEMS 1073741824ull /* 2^30; its scratch (513 KB) fits the 1 MiB array */
int pmb_inclusive_scan_u32_u64_noalloc(const uint32_t* d_in, uint64_t* d_out, size_t n, void* stream);

/* Error word of the allocation-free scan's fixed array on the current device
 * (synchronous copy, no allocation): 0 = clean; 1 = a bounded wait of the
 * last call hit its poll limit and its result is not trustworthy.  No
 * counterpart in the reference. */
int pmb_scan_noalloc_error(uint32_t* error_out);

/* Copy the error word of a scan/sort scratch buffer to the host (synchronous).
 * 0 = clean; 1 = a bounded wait hit its poll limit (a look-back, or the
 * scan's tile staging; the result is then not trustworthy).  Replaces nothing
 * in the reference (its kernels never wait on one another). */
int pmb_scratch_error(const void* d_scratch, uint32_t* error_out);

/* d_data[i] += *d_scalar for i < n (uint64; d_data 16-byte aligned, the
 * scalar read on the device).  Replaces elemAdd_cuda, the prefix sum's second
 * task (testSuite/prefixSum/source/code/src/prefixSumCUDA.cu:143-158). */
int pmb_add_u64_scalar(uint64_t* d_data, size_t n, const uint64_t* d_scalar, void* stream);

/* ------------------------------------------------------------------------ */
/* radixSort: stable LSD sort of uint32 keys                                */
/* ------------------------------------------------------------------------ */

/* Bytes of device scratch pmb_radix_sort_u32 needs (digits of 4 or 8 bits). */
size_t pmb_radix_sort_scratch_bytes(size_t n, int bits_per_pass);

/* Stable sort of d_keys[0..n) on bits [begin_bit, end_bit) (a multiple of
 * bits_per_pass, which is 4 or 8), result left in d_keys; d_alt is a second
 * device buffer of n keys.  n < 2^30; keys and scratch 16-byte aligned.  Each
 * pass is one stable counting-sort round: one round of radixSort_cpu +
 * radixSortDataRedistribution over all subtasks
 * (testSuite/radixSort/source/code/src/radixSort.cpp:55-69, :136-162;
 * the reference's GPU callback radixSort.cu:39-42 is an empty stub). */
int pmb_radix_sort_u32(uint32_t* d_keys, uint32_t* d_alt, size_t n, int begin_bit, int end_bit,
                       int bits_per_pass, void* d_scratch, size_t scratch_bytes, void* stream);

/* Stable key-value variant of pmb_radix_sort_u32: d_vals[] (n uint32 values)
 * moves with its key; d_vals_alt is the values' second buffer. */
int pmb_radix_sort_pairs_u32(uint32_t* d_keys, uint32_t* d_alt, uint32_t* d_vals, uint32_t* d_vals_alt,
                             size_t n, int begin_bit, int end_bit, int bits_per_pass, void* d_scratch,
                             size_t scratch_bytes, void* stream);

/* The digit counts (uint32, 2^bits_per_pass of them) of the first pass of the
 * last sort run with d_scratch, copied on `stream` into d_counts: the
 * per-subtask bins of a radixSort round (radixSort.cpp:127-148). */
int pmb_radix_sort_histogram(const void* d_scratch, int bits_per_pass, void* d_counts, void* stream);

/* ------------------------------------------------------------------------ */
/* pageRank: pull over CSR in-edges                                         */
/* ------------------------------------------------------------------------ */

/* Seeded R-MAT edge list (Chakrabarti et al., SDM 2004): n_edges edges over
 * 2^scale vertices, quadrant probabilities a, b, c (d = 1-a-b-c); duplicates
 * and self-loops kept; edge i depends only on (seed, i).  Stands in for the
 * reference's web-dump input, which is generated offline
 * (testSuite/pageRank/scripts/webGenerator.pl) and not shipped. */
int pmb_rmat_edges(uint64_t seed, int scale, uint64_t n_edges, double a, double b, double c,
                   uint32_t* d_src, uint32_t* d_dst, void* stream);

/* CSR by destination: row_ptr[N+1], col[E] = source of each in-edge (edges
 * of one destination keep their input order), out_degree[N].  Scratch:
 * pmb_csr_scratch_bytes; edges naming a vertex >= n_vertices are dropped and
 * set bit 2 of the scratch error word (pmb_scratch_error).  Replaces the padded fixed-stride out-link lists the
 * reference reads (pageRank.cpp:53-143). */
size_t pmb_csr_scratch_bytes(uint32_t n_vertices, uint64_t n_edges);
int pmb_csr_by_destination(const uint32_t* d_src, const uint32_t* d_dst, uint32_t n_vertices, uint64_t n_edges,
                           uint32_t* d_row_ptr, uint32_t* d_col, uint32_t* d_out_degree, void* d_scratch,
                           size_t scratch_bytes, void* stream);

/* The reference's web-dump pages (pageRank.cpp:53-111, the page files
 * mapped by pmMapFiles and read by pageRank_cpu / pageRank_cudaLaunchFunc):
 * per page a u32 out-link count, then max_outlinks u32 slots whose first
 * `count` hold 1-based target ids; pages max_outlinks + 1 words apart.
 *
 * pmb_csr_from_webdump: n_pages pages (sources 0..n_pages-1, n_pages <=
 * n_vertices) -> CSR by destination over n_vertices rows, as
 * pmb_csr_by_destination builds it (edges of one destination in page order).
 * n_edges must be the sum of the counts.  Error word of d_scratch
 * (pmb_scratch_error): bit 2 a target outside [1, n_vertices] (dropped) or a
 * slot left unfilled, bit 4 a count above max_outlinks (clamped), bit 8 more
 * edges than n_edges (dropped).  Replaces readWebPagesFile +
 * the padded device copy of singleGpuPageRank (pageRankCUDA.cu:166-190). */
size_t pmb_webdump_csr_scratch_bytes(uint32_t n_pages, uint32_t n_vertices, uint64_t n_edges);
int pmb_csr_from_webdump(const uint32_t* d_dump, uint32_t n_pages, uint32_t max_outlinks, uint32_t n_vertices,
                         uint64_t n_edges, uint32_t* d_row_ptr, uint32_t* d_col, uint32_t* d_out_degree,
                         void* d_scratch, size_t scratch_bytes, void* stream);

/* One push step of the reference over n_pages device-resident web-dump pages
 * (zeroInit + pageRank_cuda, pageRankCUDA.cu:46-76): d_out[0..n_vertices) is
 * zeroed, then every page with count > 0 adds (damping * r) / count to each of
 * its targets, r = d_rank_in[page] or initial_rank when d_rank_in is NULL.
 * fp32 adds in L2 in no fixed order (as the reference's atomics).  A target
 * outside [1, n_vertices] is skipped and a count above max_outlinks clamped;
 * either sets bit 2 of *d_err when d_err is not NULL. */
int pmb_webdump_push(const uint32_t* d_dump, uint32_t n_pages, uint32_t max_outlinks, const float* d_rank_in,
                     float initial_rank, float damping, float* d_out, uint32_t n_vertices, uint32_t* d_err,
                     void* stream);

/* Edge-slice partition of a CSR graph (once per graph). */
size_t pmb_pagerank_plan_bytes(uint32_t n_vertices, uint64_t n_edges);
int pmb_pagerank_plan(const uint32_t* d_row_ptr, uint32_t n_vertices, uint64_t n_edges, void* d_plan,
                      size_t plan_bytes, void* stream);

/* `iterations` PageRank steps r'[v] = sum_{u->v} damping*r[u]/outdeg(u) (no
 * teleport), fp32, starting from d_rank_in, final ranks in d_rank_out.
 * d_work: pmb_pagerank_work_bytes.  Replaces pageRank_cudaLaunchFunc /
 * pageRank_cuda / zeroInit (testSuite/pageRank/source/code/src/
 * pageRankCUDA.cu:46-164) plus the host REDUCE_ADD of the subtasks' rank
 * arrays (pageRank.cpp:554-555); equals pageRank_cpu (:336-378) up to fp32
 * summation order.  Each rank has a single writer: results are deterministic. */
size_t pmb_pagerank_work_bytes(uint32_t n_vertices, uint64_t n_edges);
int pmb_pagerank(const uint32_t* d_row_ptr, const uint32_t* d_col, const uint32_t* d_out_degree, uint32_t n_vertices,
                 uint64_t n_edges, const void* d_plan, float damping, int iterations, const float* d_rank_in,
                 float* d_rank_out, void* d_work, size_t work_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* matrixMultiply / luDecomposition: fp32 GEMM on tcgen05 tensor cores       */
/* ------------------------------------------------------------------------ */

/* Device workspace (256-byte aligned) pmb_sgemm_bf16x3 needs for M x N x K. */
size_t pmb_gemm_workspace_bytes(int M, int N, int K);

/* Row-major C = alpha*A*B + beta*C with fp32 operands (A: M x K, lda; B:
 * K x N, ldb; C: M x N, ldc; all device pointers), computed as a BF16x3
 * split product (A = Ahi + Alo, B = Bhi + Blo; Ahi*Bhi + Ahi*Blo + Alo*Bhi)
 * with FP32 accumulation in tensor memory.  One split launch pair and one
 * GEMM launch on `stream`.  Word 1 of the workspace is an error word
 * (pmb_scratch_error): value 4 = a pipeline wait expired.  Replaces the
 * cublasSgemm calls of matrixMultiply_cudaLaunchFunc
 * (testSuite/matrixMultiplyBlas/source/code/src/matrixMultiplyBlasCUDA.cu:54-77)
 * and diagComp_cudaLaunchFunc (luDecompositionCUDA.cu:153-193); for column-
 * major data call it with the operands swapped (C^T = B^T A^T). */
int pmb_sgemm_bf16x3(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                     float beta, float* C, int64_t ldc, void* workspace, size_t ws_bytes, void* stream);

/* One product of a grouped call: C = alpha*A*B + beta*C, row-major fp32
 * device operands as in pmb_sgemm_bf16x3. */
typedef struct pmb_gemm_problem {
    int M, N, K;
    float alpha;
    const float* A;
    int64_t lda;
    const float* B;
    int64_t ldb;
    float beta;
    float* C;
    int64_t ldc;
} pmb_gemm_problem;

/* Device workspace (256-byte aligned) pmb_sgemm_bf16x3_grouped needs for
 * `count` problems. */
size_t pmb_gemm_grouped_workspace_bytes(const pmb_gemm_problem* problems, int count);

/* `count` independent BF16x3 products of different shapes (each with the
 * arithmetic of pmb_sgemm_bf16x3) in one launch of the product kernel per 24
 * products, after one split launch per product: the tiles of all products
 * go to the CTA pairs of one grid, so small products share the GPU instead
 * of each filling a launch of its own.  `problems` is a host array; the
 * products must not overlap in C.  Word 1 of the workspace is the error word
 * (pmb_scratch_error).  No counterpart in the reference, whose subtasks each
 * call cublasSgemm (matrixMultiplyBlasCUDA.cu:54-77); the runtime's batch
 * hook of the matrixMultiplyBlas app calls it for all subtasks of a task. */
int pmb_sgemm_bf16x3_grouped(const pmb_gemm_problem* problems, int count, void* workspace, size_t workspace_bytes,
                             void* stream);

/* Plain GPU form of the same product: FP32 SIMT, 64 x 64 shared-memory
 * tiles, no tensor cores (the one-task-at-a-time FP32 baseline). */
int pmb_sgemm_plain(int M, int N, int K, float alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                    float beta, float* C, int64_t ldc, void* stream);

/* ------------------------------------------------------------------------ */
/* luDecomposition: blocked unpivoted LU (Crout form), column-major          */
/* ------------------------------------------------------------------------ */

/* Device workspace (256-byte aligned) for an n x n LU with block size nb. */
size_t pmb_lu_workspace_bytes(int n, int nb);

/* In-place LU of the column-major n x n fp32 matrix d_A (lda >= n) in the
 * reference's form: L lower triangular WITH the pivots on its diagonal, U unit
 * upper triangular, A = L*U, no row exchanges
 * (testSuite/luDecomposition/source/code/src/luDecomposition.cpp:116-125).
 * Block size nb in [1,128].  Replaces the three task stages
 * luDecomposition_cudaLaunchFunc / horizVertComp_cudaLaunchFunc /
 * diagComp_cudaLaunchFunc (luDecompositionCUDA.cu:66-193): the nb x nb
 * diagonal blocks are factored in FP64, the panels are solved in FP64 from
 * those factors (nb <= 64; larger blocks use FP64 inverses and BF16x3 GEMMs)
 * and the trailing updates run as BF16x3 tensor-core GEMMs.  Word 1 of the
 * workspace gets flags (pmb_scratch_error): 1 = partial pivoting (FP64
 * comparison) would have exchanged rows in some column, 2 = a zero pivot,
 * 4 = a kernel's bounded wait expired (the result is not valid).  For
 * nb <= 64 the serial chain of each step (diagonal block, panels, the next
 * block column of the update) runs on a high-priority stream the library
 * keeps per (device, `stream`) while the rest of the update runs on `stream`
 * (PMB_LU_LOOKAHEAD=0: everything on `stream`); calls that share `stream`
 * must come from one host thread at a time. */
int pmb_lu_decompose(float* d_A, int n, int64_t lda, int nb, void* d_workspace, size_t ws_bytes, void* stream);

/* Same factorization with FP32 SIMT GEMMs (the plain one-task-at-a-time form). */
int pmb_lu_decompose_plain(float* d_A, int n, int64_t lda, int nb, void* d_workspace, size_t ws_bytes,
                           void* stream);

/* Triangular solve in place, fp32 column-major, no transpose, alpha = 1:
 *   side PMB_SIDE_LEFT,  uplo PMB_FILL_LOWER: B <- L^-1 B (L = the m x m lower
 *     triangle of d_A, B m x n);
 *   side PMB_SIDE_RIGHT, uplo PMB_FILL_UPPER: B <- B U^-1 (U = the n x n upper
 *     triangle of d_A, B m x n);
 * diag PMB_DIAG_UNIT ignores the stored diagonal.  64-wide diagonal blocks are
 * solved in FP64, the remaining rows (left) or columns (right) are updated by
 * BF16x3 tensor-core GEMMs.  d_workspace: pmb_trsm_workspace_bytes(side, m, n)
 * bytes, 256-byte aligned.  Replaces cublasStrsm in horizVertComp_cudaLaunchFunc
 * (testSuite/luDecomposition/source/code/src/luDecompositionCUDA.cu:99-151:
 * left/lower/non-unit for U01 = L00^-1 A01, right/upper/unit for
 * L10 = A10 U00^-1). */
#define PMB_SIDE_LEFT 0
#define PMB_SIDE_RIGHT 1
#define PMB_FILL_LOWER 0
#define PMB_FILL_UPPER 1
#define PMB_DIAG_NON_UNIT 0
#define PMB_DIAG_UNIT 1
size_t pmb_trsm_workspace_bytes(int side, int m, int n);
int pmb_trsm_f32(int side, int uplo, int diag, int m, int n, const float* d_A, int64_t lda, float* d_B, int64_t ldb,
                 void* d_workspace, size_t ws_bytes, void* stream);

/* FP64 residual: d_sums[0] = ||A0 - L*U||_F^2, d_sums[1] = ||A0||_F^2 (two
 * device doubles), L and U read from the packed factorization d_LU. */
int pmb_lu_residual_f64(const float* d_A0, int64_t lda0, const float* d_LU, int64_t ldlu, int n, double* d_sums,
                        void* stream);

/* FP64 refinement of a solve with fp32 LU factors: A x = b for the n x n
 * column-major d_A0 (fp32, lda0) factored into d_LU by pmb_lu_decompose
 * (Crout form, ldlu).  x_0 = U^-1 L^-1 b, then `iterations` steps of
 * r = b - A x in FP64, x += U^-1 L^-1 r, all triangular solves in FP64.
 * d_b, d_x: n device doubles; d_berr: iterations + 1 device doubles receiving
 * the normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf +
 * ||b||_inf) after each solve.  d_workspace: pmb_lu_refine_workspace_bytes(n).
 * No counterpart in the reference, whose LU stays in fp32
 * (luDecomposition.cpp:116-125); it is the FP64 residual / refinement step
 * of the split-precision LU. */
size_t pmb_lu_refine_workspace_bytes(int n);
int pmb_lu_solve_refined(const float* d_A0, int64_t lda0, const float* d_LU, int64_t ldlu, int n, const double* d_b,
                         double* d_x, int iterations, double* d_berr, void* d_workspace, size_t ws_bytes,
                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PMB_CAPI_H */
