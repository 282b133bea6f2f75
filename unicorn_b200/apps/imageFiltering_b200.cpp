// B200 GPU callbacks of the imageFiltering app: a drop-in replacement for
// testSuite/imageFiltering/source/code/src/imageFilteringCUDA.cu (whose
// texture-reference kernel no longer compiles with CUDA 12).
//
// imageFilter_cudaLaunchFunc keeps the reference callback's contract
// (:295-342): the subtask's rectangle comes from the app's
// GetSubtaskSubscription, the input view is the clamped tile + halo of the
// bottom-up image and the output view the tile, each NATURAL (row pitch 3W) or
// COMPACT (packed rows).  It enqueues one stencil launch on the subtask's
// stream and allocates nothing, so no reserved device memory is requested.
// A batch hook lets the runtime run all subtasks of a task (NATURAL views) as
// one launch of the same kernel.
#include "imageFiltering_b200.h"

#include <cstring>
#include <vector>

#include "pmb_capi.h"

extern "C" int pmb_runtime_register_batch(void* subtask_gpu_custom, void* batch_fn);

namespace imageFiltering {

using namespace pm;

namespace {

bool item_for(imageFilterTaskConf* conf, const pmSubtaskInfo& si, pmb_imgf_item& it) {
    int c0, c1, r0, r1;
    pmSplitInfo split = si.splitInfo;
    if (!GetSubtaskSubscription(conf, si.subtaskId, split, &c0, &c1, &r0, &r1)) return false;
    const int W = static_cast<int>(conf->imageWidth), H = static_cast<int>(conf->imageHeight);
    const int R = static_cast<int>(conf->filterRadius);
    const int last_row = r1 - 1 + R >= H ? H - 1 : r1 - 1 + R;
    const int first_col = c0 - R < 0 ? 0 : c0 - R;
    const int last_col = c1 - 1 + R >= W ? W - 1 : c1 - 1 + R;
    const pmMemInfo& in = si.memInfo[kInputMemIndex];
    const pmMemInfo& out = si.memInfo[kOutputMemIndex];
    it.in = static_cast<const uint8_t*>(in.ptr);
    it.out = static_cast<uint8_t*>(out.ptr);
    it.in_pitch = in.visibilityType == SUBSCRIPTION_NATURAL ? 3LL * W : 3LL * (last_col - first_col + 1);
    it.out_pitch = out.visibilityType == SUBSCRIPTION_NATURAL ? 3LL * W : 3LL * (c1 - c0);
    it.width = W;
    it.height = H;
    it.in_row0 = H - 1 - last_row;
    it.in_col0 = first_col;
    it.out_row0 = r0;
    it.out_col0 = c0;
    it.r0 = r0;
    it.r1 = r1;
    it.c0 = c0;
    it.c1 = c1;
    return true;
}

pmStatus to_pm(int st) { return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st); }

// All subtasks of one task in one launch (chunks of PMB_IMGF_MAX_ITEMS).
pmStatus imageFilter_batch(const pmTaskInfo* task, const pmDeviceInfo*, const pmSubtaskInfo* subtasks,
                           unsigned long count, void* stream) {
    imageFilterTaskConf* conf = static_cast<imageFilterTaskConf*>(task->taskConf);
    std::vector<pmb_imgf_item> items;
    items.reserve(count);
    for (unsigned long i = 0; i < count; ++i) {
        pmb_imgf_item it;
        if (item_for(conf, subtasks[i], it)) items.push_back(it);
    }
    for (size_t b = 0; b < items.size(); b += PMB_IMGF_MAX_ITEMS) {
        const int n = static_cast<int>(items.size() - b < PMB_IMGF_MAX_ITEMS ? items.size() - b : PMB_IMGF_MAX_ITEMS);
        const int st = pmb_image_filter(items.data() + b, n, reinterpret_cast<const int8_t*>(conf->filter),
                                        static_cast<int>(conf->filterRadius), PMB_IMGF_WRAP, stream);
        if (st != PMB_SUCCESS) return to_pm(st);
    }
    return pmSuccess;
}

struct Registrar {
    Registrar() {
        pmb_runtime_register_batch(reinterpret_cast<void*>(&imageFilter_cudaLaunchFunc),
                                   reinterpret_cast<void*>(&imageFilter_batch));
    }
} g_registrar;

}  // namespace

size_t computeSubtaskReservedMemRequirement(pmTaskInfo, pmDeviceInfo, unsigned long, int, int, int, int) {
    return 0;  // the stencil reads the subscription views directly: no staging copy, no filter upload
}

pmStatus imageFilter_cudaLaunchFunc(pmTaskInfo pTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream) {
    imageFilterTaskConf* conf = static_cast<imageFilterTaskConf*>(pTaskInfo.taskConf);
    pmb_imgf_item it;
    if (!item_for(conf, pSubtaskInfo, it)) return pmSuccess;
    return to_pm(pmb_image_filter(&it, 1, reinterpret_cast<const int8_t*>(conf->filter),
                                  static_cast<int>(conf->filterRadius), PMB_IMGF_WRAP, pCudaStream));
}

int singleGpuImageFilter(void* pInvertedImageData, size_t pImageWidth, size_t pImageHeight,
                         char pFilter[kMaxFilterDim][kMaxFilterDim], size_t pFilterRadius, size_t pImageBytesPerLine,
                         void* pOutputMem) {
    const size_t bytes = pImageWidth * pImageHeight * kPixelCount;
    if (pImageBytesPerLine != pImageWidth * kPixelCount) return 1;
    void *d_in = nullptr, *d_out = nullptr, *s = nullptr;
    int st = pmb_malloc(&d_in, bytes);
    if (st == PMB_SUCCESS) st = pmb_malloc(&d_out, bytes);
    if (st == PMB_SUCCESS) st = pmb_stream_create(&s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(d_in, pInvertedImageData, bytes, PMB_H2D, s);
    if (st == PMB_SUCCESS)
        st = pmb_image_filter_full(static_cast<const uint8_t*>(d_in), static_cast<uint8_t*>(d_out),
                                   static_cast<int>(pImageWidth), static_cast<int>(pImageHeight),
                                   reinterpret_cast<const int8_t*>(pFilter), static_cast<int>(pFilterRadius),
                                   PMB_IMGF_WRAP, s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(pOutputMem, d_out, bytes, PMB_D2H, s);
    if (st == PMB_SUCCESS) st = pmb_stream_synchronize(s);
    pmb_stream_destroy(s);
    pmb_free(d_in);
    pmb_free(d_out);
    return st == PMB_SUCCESS ? 0 : 1;
}

}  // namespace imageFiltering
