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

/* Whole-image convenience form: one item covering the full image with
 * NATURAL views (in_pitch = out_pitch = 3W). */
int pmb_image_filter_full(const uint8_t* d_in, uint8_t* d_out, int width, int height,
                          const int8_t* filter, int radius, int mode, void* stream);

/* Plain GPU form: one thread per output pixel, 3*(2r+1)^2 byte loads from
 * global memory and scalar multiply-adds; NATURAL views only.  The
 * one-task-at-a-time baseline the stencil kernel is compared with. */
int pmb_image_filter_plain(const uint8_t* d_in, uint8_t* d_out, int width, int height,
                           const int8_t* filter, int radius, int mode, void* stream);

/* ------------------------------------------------------------------------ */
/* prefixSum: inclusive scan                                                */
/* ------------------------------------------------------------------------ */

/* Bytes of device scratch pmb_inclusive_scan_u32_u64 needs for n elements
 * (a 256-byte header plus 8 bytes per 4096-element tile). */
size_t pmb_scan_scratch_bytes(size_t n);

/* out[i] = in[0] + ... + in[i] with 64-bit sums, n <= 2^30, one launch on
 * `stream` (plus a memset of the scratch).  d_in, d_out and d_scratch are
 * device pointers, 16-byte aligned.  Replaces prefixSum_cudaLaunchFunc /
 * prefixSum_cuda / elemAdd_cuda and the host scan of subtask totals
 * (testSuite/prefixSum/source/code/src/prefixSumCUDA.cu:68-267,
 * prefixSum.cpp:189-294); result equals serialPrefixSum (prefixSum.cpp:47-53)
 * widened to uint64. */
int pmb_inclusive_scan_u32_u64(const uint32_t* d_in, uint64_t* d_out, size_t n, void* d_scratch,
                               size_t scratch_bytes, void* stream);

/* Copy the error word of a scan/sort scratch buffer to the host (synchronous).
 * 0 = clean; 1 = a look-back wait hit its poll limit (the result is then
 * not trustworthy).  Replaces nothing in the reference (its kernels never wait
 * on one another). */
int pmb_scratch_error(const void* d_scratch, uint32_t* error_out);

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

#ifdef __cplusplus
}
#endif

#endif /* PMB_CAPI_H */
