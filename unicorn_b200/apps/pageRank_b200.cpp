// B200 GPU callbacks of the pageRank app: a drop-in replacement for
// testSuite/pageRank/source/code/src/pageRankCUDA.cu.
//
// pageRank_cudaLaunchFunc keeps the reference callback's contract
// (:119-164): the subtask's pages are those of the app's data distribution
// (pageRank.cpp:278-307), their page files come from the app's
// LoadMappedFiles and are copied into the subtask's reserved device memory
// (pmReserveCudaGlobalMem, sized by the app), and one push step writes the
// subtask's copy of the whole rank array, which the runtime folds across
// subtasks with the app's REDUCE_ADD callback (on the device).
//
// singleGpuPageRank (:166-209) builds the graph once as CSR in-edges from the
// whole padded dump (pmb_csr_from_webdump) and runs the deterministic pull
// iterations (pmb_pagerank) instead of re-pushing with atomics.
#include "pageRank_b200.h"

#include <cstring>
#include <vector>

#include "pmb_capi.h"

namespace pageRank {

using namespace pm;

namespace {

pmStatus to_pm(int st) { return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st); }

// pageRankCUDA.cu:124-127: pages of a subtask and its page files.
unsigned int pages_of(const pageRankTaskConf* c, unsigned long id) {
    const unsigned long end = (id + 1) * c->webPagesPerSubtask;
    return static_cast<unsigned int>(c->totalWebPages < end ? c->totalWebPages - id * c->webPagesPerSubtask
                                                            : c->webPagesPerSubtask);
}

}  // namespace

pmStatus pageRank_cudaLaunchFunc(pmTaskInfo pTaskInfo, pmDeviceInfo, pmSubtaskInfo pSubtaskInfo, void* pCudaStream) {
    pageRankTaskConf* conf = static_cast<pageRankTaskConf*>(pTaskInfo.taskConf);
    const unsigned long id = pSubtaskInfo.subtaskId;
    const unsigned int pages = pages_of(conf, id);
    const unsigned int per_file = conf->webPagesPerFile;
    const unsigned int files = pages / per_file + (pages % per_file ? 1 : 0);
    const unsigned int first = static_cast<unsigned int>(id) * files;
    const unsigned int total_files = conf->totalWebPages / per_file + (conf->totalWebPages % per_file ? 1 : 0);
    const size_t stride = static_cast<size_t>(conf->maxOutlinksPerWebPage) + 1;
    unsigned int* dump = static_cast<unsigned int*>(pSubtaskInfo.gpuContext.reservedGlobalMem);
    if (!dump || !conf->maxOutlinksPerWebPage) return pmDataProcessingFailure;

    // The subtask's pages, file by file, into the reserved memory (the app
    // reserved pages * stride words); never more pages than the subtask has.
    void** ptrs = LoadMappedFiles(conf, id);
    unsigned int copied = 0;
    int st = PMB_SUCCESS;
    for (unsigned int i = 0; i < files && st == PMB_SUCCESS && copied < pages; ++i) {
        unsigned int in_file = per_file;
        if (i + first == total_files - 1) in_file = conf->totalWebPages - (i + first) * per_file;
        if (in_file > pages - copied) in_file = pages - copied;
        if (!ptrs[i]) {
            st = PMB_INVALID_INDEX;
            break;
        }
        st = pmb_memcpy_async(dump + copied * stride, ptrs[i], static_cast<size_t>(in_file) * stride * 4, PMB_H2D,
                              pCudaStream);
        copied += in_file;
    }
    delete[] ptrs;
    if (st != PMB_SUCCESS) return to_pm(st);

    const float* rank_in =
        conf->iteration == 0 ? nullptr : static_cast<const float*>(pSubtaskInfo.memInfo[kInputMemIndex].ptr);
    float* out = static_cast<float*>(pSubtaskInfo.memInfo[kOutputMemIndex].ptr);
    return to_pm(pmb_webdump_push(dump, copied, conf->maxOutlinksPerWebPage, rank_in, conf->initialPageRank,
                                  kDampeningFactor, out, conf->totalWebPages, nullptr, pCudaStream));
}

int singleGpuPageRank(pageRankTaskConf& pTaskConf, unsigned int* pWebDump, void* pOutputMem) {
    const uint32_t n = pTaskConf.totalWebPages, maxo = pTaskConf.maxOutlinksPerWebPage;
    if (!n || !maxo) return 1;
    const size_t stride = static_cast<size_t>(maxo) + 1;
    uint64_t edges = 0;
    for (uint32_t p = 0; p < n; ++p) {
        const uint32_t c = pWebDump[p * stride];
        edges += c < maxo ? c : maxo;
    }
    void *s = nullptr, *d_dump = nullptr, *row_ptr = nullptr, *col = nullptr, *deg = nullptr, *scratch = nullptr;
    void *plan = nullptr, *work = nullptr, *r0 = nullptr, *r1 = nullptr;
    const size_t scratch_bytes = pmb_webdump_csr_scratch_bytes(n, n, edges);
    const size_t plan_bytes = pmb_pagerank_plan_bytes(n, edges);
    const size_t work_bytes = pmb_pagerank_work_bytes(n, edges);
    int st = pmb_stream_create(&s);
    if (st == PMB_SUCCESS) st = pmb_malloc(&d_dump, n * stride * 4);
    if (st == PMB_SUCCESS) st = pmb_malloc(&row_ptr, 4ull * (n + 1));
    if (st == PMB_SUCCESS) st = pmb_malloc(&col, 4 * (edges ? edges : 1));
    if (st == PMB_SUCCESS) st = pmb_malloc(&deg, 4ull * n);
    if (st == PMB_SUCCESS) st = pmb_malloc(&scratch, scratch_bytes);
    if (st == PMB_SUCCESS) st = pmb_malloc(&plan, plan_bytes);
    if (st == PMB_SUCCESS) st = pmb_malloc(&work, work_bytes);
    if (st == PMB_SUCCESS) st = pmb_malloc(&r0, 4ull * n);
    if (st == PMB_SUCCESS) st = pmb_malloc(&r1, 4ull * n);
    std::vector<float> init(n, pTaskConf.initialPageRank);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(d_dump, pWebDump, n * stride * 4, PMB_H2D, s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(r0, init.data(), 4ull * n, PMB_H2D, s);
    if (st == PMB_SUCCESS)
        st = pmb_csr_from_webdump(static_cast<const uint32_t*>(d_dump), n, maxo, n, edges,
                                  static_cast<uint32_t*>(row_ptr), static_cast<uint32_t*>(col),
                                  static_cast<uint32_t*>(deg), scratch, scratch_bytes, s);
    if (st == PMB_SUCCESS)
        st = pmb_pagerank_plan(static_cast<const uint32_t*>(row_ptr), n, edges, plan, plan_bytes, s);
    if (st == PMB_SUCCESS)
        st = pmb_pagerank(static_cast<const uint32_t*>(row_ptr), static_cast<const uint32_t*>(col),
                          static_cast<const uint32_t*>(deg), n, edges, plan, kDampeningFactor, kPageRankIterations,
                          static_cast<const float*>(r0), static_cast<float*>(r1), work, work_bytes, s);
    if (st == PMB_SUCCESS) st = pmb_memcpy_async(pOutputMem, r1, 4ull * n, PMB_D2H, s);
    if (st == PMB_SUCCESS) st = pmb_stream_synchronize(s);
    uint32_t err = 0;
    if (st == PMB_SUCCESS) st = pmb_scratch_error(scratch, &err);
    for (void* p : {d_dump, row_ptr, col, deg, scratch, plan, work, r0, r1})
        if (p) pmb_free(p);
    if (s) pmb_stream_destroy(s);
    return st == PMB_SUCCESS && err == 0 ? 0 : 1;
}

}  // namespace pageRank
