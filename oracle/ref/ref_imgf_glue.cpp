/*
 * ref_imgf_glue.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Drives the reference's own imageFiltering CPU callbacks
 * (testSuite/imageFiltering/source/code/src/imageFiltering.cpp, compiled
 * unchanged from the reference tree by oracle/ref/Makefile) outside the
 * reference runtime, so tests and the CPU baseline can run them on seeded
 * inputs:
 *   - imageFilterDataDistribution (:342-377) is called for each subtask; the
 *     pmSubscribeToMemory calls it makes are recorded here, exactly as the
 *     runtime's subscription manager would, and turned into NATURAL-view
 *     pointers (address-space base + subscription offset);
 *   - imageFilter_cpu (:379-472) then runs on those pointers.
 * Subtasks (and, optionally, row splits of each subtask -- the reference's
 * canSplitCpuSubtasks mechanism, GetSubtaskSubscription :319-337) are pulled
 * by a pool of worker threads, one per requested core, mirroring the
 * reference's one CPU execution stub per core.
 *
 * The commonAPI functions and pm:: calls the app file references but the
 * callbacks never reach are stubbed below.
 */
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "commonAPI.h"
#include "imageFiltering.h"

namespace {
struct Recorded {
    bool valid[pm::MAX_MEM_SECTIONS_PER_TASK];
    pm::pmScatteredSubscriptionInfo info[pm::MAX_MEM_SECTIONS_PER_TASK];
};
thread_local Recorded t_rec;
}  // namespace

namespace pm {
pmStatus pmSubscribeToMemory(pmTaskHandle, pmDeviceHandle, ulong, pmSplitInfo&, uint pMemIndex,
                             pmSubscriptionType, const pmScatteredSubscriptionInfo& pInfo) {
    if (pMemIndex >= MAX_MEM_SECTIONS_PER_TASK) return pmInvalidIndex;
    t_rec.valid[pMemIndex] = true;
    t_rec.info[pMemIndex] = pInfo;
    return pmSuccess;
}
pmStatus pmSubmitTask(pmTaskDetails, pmTaskHandle*) { return pmStatusUnavailable; }
pmStatus pmFetchMemory(pmMemHandle) { return pmStatusUnavailable; }
pmStatus pmReleaseTask(pmTaskHandle) { return pmStatusUnavailable; }
pmStatus pmGetRawMemPtr(pmMemHandle, pmRawMemPtr*) { return pmStatusUnavailable; }
pmStatus pmReleaseMemory(pmMemHandle) { return pmStatusUnavailable; }
pmStatus pmCreateMemory2D(size_t, size_t, pmMemHandle*) { return pmStatusUnavailable; }
pmStatus pmWaitForTaskCompletion(pmTaskHandle) { return pmStatusUnavailable; }
}  // namespace pm

void commonStart(int, char**, initFunc, serialProcessFunc, singleGpuProcessFunc, parallelProcessFunc,
                 compareFunc, destroyFunc, callbackStruct*, size_t) {}
void commonFinish() {}
void DistributeMemory(pmMemHandle, memDistributionType, unsigned int, unsigned int, unsigned int,
                      unsigned int, bool) {}
uint getAffinityCriterion() { return 0; }
double getCurrentTimeInSecs() { return 0.0; }
bool isMultiAssignEnabled() { return false; }
bool isComputeCommunicationOverlapEnabled() { return false; }

namespace imageFiltering {
pmStatus imageFilterDataDistribution(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
pmStatus imageFilter_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo);
}  // namespace imageFiltering

namespace {
using namespace imageFiltering;

void make_conf(imageFilterTaskConf* conf, int W, int H, int R, const int8_t* filter) {
    std::memset(conf, 0, sizeof(*conf));
    conf->imageWidth = W;
    conf->imageHeight = H;
    conf->imageOffset = 0;
    conf->imageBytesPerLine = (size_t)W * PIXEL_COUNT;
    conf->filterRadius = R;
    for (int i = 0; i < MAX_FILTER_DIM; ++i)
        for (int j = 0; j < MAX_FILTER_DIM; ++j) conf->filter[i][j] = (char)filter[i * MAX_FILTER_DIM + j];
}

unsigned long subtask_count(int W, int H) {
    const unsigned long tx = W / TILE_DIM + (W % TILE_DIM ? 1 : 0);
    const unsigned long ty = H / TILE_DIM + (H % TILE_DIM ? 1 : 0);
    return tx * ty;
}

int run_one(imageFilterTaskConf* conf, unsigned long nsub, const uint8_t* in, uint8_t* out,
            unsigned long id, unsigned split_id, unsigned split_count) {
    pmTaskInfo ti;
    ti.taskConf = conf;
    ti.taskConfLength = sizeof(*conf);
    ti.subtaskCount = nsub;
    pmDeviceInfo di;
    di.deviceType = pm::CPU;
    pmSubtaskInfo si;
    si.subtaskId = id;
    si.splitInfo = pmSplitInfo(split_id, split_count);
    std::memset(&t_rec, 0, sizeof(t_rec));
    if (imageFilterDataDistribution(ti, di, si) != pmSuccess) return 1;
    if (!t_rec.valid[OUTPUT_MEM_INDEX]) return 0;  // split with no rows: nothing to do
    if (!t_rec.valid[INPUT_MEM_INDEX]) return 2;
    si.memCount = MAX_MEM_INDICES;
    si.memInfo[INPUT_MEM_INDEX] = pmMemInfo((void*)(in + t_rec.info[INPUT_MEM_INDEX].offset),
                                            (void*)(in + t_rec.info[INPUT_MEM_INDEX].offset), NULL,
                                            0, SUBSCRIPTION_NATURAL);
    si.memInfo[OUTPUT_MEM_INDEX] = pmMemInfo((void*)(out + t_rec.info[OUTPUT_MEM_INDEX].offset), NULL,
                                             (void*)(out + t_rec.info[OUTPUT_MEM_INDEX].offset), 0,
                                             SUBSCRIPTION_NATURAL);
    return imageFilter_cpu(ti, di, si) == pmSuccess ? 0 : 3;
}
}  // namespace

extern "C" {

/* Reference tile edge (TILE_DIM of imageFiltering.h) this library was compiled with. */
int ref_imgf_tile_dim(void) { return TILE_DIM; }

/* Number of subtasks the reference would create for a W x H image. */
unsigned long ref_imgf_subtask_count(int W, int H) { return subtask_count(W, H); }

/* Subscriptions the reference's data-distribution callback makes for one
 * subtask: out[0..3] = input {offset,size,step,count}, out[4..7] = output. */
int ref_imgf_subscriptions(int W, int H, int R, unsigned long id, unsigned long long* out8) {
    imageFilterTaskConf conf;
    int8_t zero[MAX_FILTER_DIM * MAX_FILTER_DIM] = {0};
    make_conf(&conf, W, H, R, zero);
    pmTaskInfo ti;
    ti.taskConf = &conf;
    ti.subtaskCount = subtask_count(W, H);
    pmDeviceInfo di;
    di.deviceType = pm::CPU;
    pmSubtaskInfo si;
    si.subtaskId = id;
    std::memset(&t_rec, 0, sizeof(t_rec));
    if (imageFilterDataDistribution(ti, di, si) != pmSuccess) return 1;
    for (int k = 0; k < 2; ++k) {
        const pmScatteredSubscriptionInfo& s = t_rec.info[k];
        out8[4 * k + 0] = s.offset;
        out8[4 * k + 1] = s.size;
        out8[4 * k + 2] = s.step;
        out8[4 * k + 3] = s.count;
    }
    return 0;
}

/* Run every subtask of the task over `threads` workers; each subtask is cut
 * into `split` row slices (split <= 1: no splitting).  Returns 0 on success. */
int ref_imgf_task(const uint8_t* in, uint8_t* out, int W, int H, int R, const int8_t* filter,
                  int threads, int split) {
    imageFilterTaskConf conf;
    make_conf(&conf, W, H, R, filter);
    const unsigned long nsub = subtask_count(W, H);
    const unsigned sc = split > 1 ? (unsigned)split : 0u;
    const unsigned long units = nsub * (sc ? sc : 1);
    std::atomic<unsigned long> next(0);
    std::atomic<int> err(0);
    auto worker = [&]() {
        for (;;) {
            const unsigned long u = next.fetch_add(1);
            if (u >= units) break;
            const unsigned long id = sc ? u / sc : u;
            const unsigned sid = sc ? (unsigned)(u % sc) : 0u;
            const int st = run_one(&conf, nsub, in, out, id, sid, sc);
            if (st) err.store(st);
        }
    };
    if (threads < 1) threads = 1;
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return err.load();
}

}  // extern "C"
