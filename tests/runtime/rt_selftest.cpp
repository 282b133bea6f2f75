// Self-test of the pm:: runtime (libpmlib.so) through its public API.
// Usage: rt_selftest <test> [args]; prints "PASS <test>" and exits 0, or
// prints "FAIL <test>: <reason>" and exits 1.  The GPU tests need a device;
// the CPU tests force CPU execution by registering no GPU callback.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "pmPublicDefinitions.h"
#include "pmb_capi.h"

using namespace pm;

extern "C" void* rt_add_kernel_ptr();
extern "C" void pmb_runtime_stats(unsigned long long*, unsigned long long*, unsigned long long*, unsigned long long*);
extern "C" void pmb_runtime_reset_stats(void);

namespace {

std::string g_test;
#define CHECK(cond, ...)                                   \
    do {                                                   \
        if (!(cond)) {                                     \
            std::printf("FAIL %s: ", g_test.c_str());      \
            std::printf(__VA_ARGS__);                      \
            std::printf(" [%s]\n", pmGetLastError());      \
            std::exit(1);                                  \
        }                                                  \
    } while (0)

struct RtConf {
    int add;
    int ld;
};

constexpr int kRows = 300, kCols = 257, kTile = 64;

int tiles_x() { return (kCols + kTile - 1) / kTile; }
int tiles() { return tiles_x() * ((kRows + kTile - 1) / kTile); }
void tile_of(unsigned long id, int& r0, int& r1, int& c0, int& c1) {
    r0 = static_cast<int>(id / tiles_x()) * kTile;
    c0 = static_cast<int>(id % tiles_x()) * kTile;
    r1 = std::min(r0 + kTile, kRows);
    c1 = std::min(c0 + kTile, kCols);
}

int g_extra = 5;
pmStatus g_sub_status = pmSuccess;  // first non-success subscription status seen

pmStatus add_dd(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    int r0, r1, c0, c1;
    tile_of(si.subtaskId, r0, r1, c0, c1);
    const pmScatteredSubscriptionInfo s((size_t(r0) * kCols + c0) * 4, size_t(c1 - c0) * 4, size_t(kCols) * 4,
                                        size_t(r1 - r0));
    pmStatus a = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION, s);
    pmStatus b = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, WRITE_SUBSCRIPTION, s);
    if (a != pmSuccess && g_sub_status == pmSuccess) g_sub_status = a;
    if (b != pmSuccess && g_sub_status == pmSuccess) g_sub_status = b;
    int* sc = static_cast<int*>(pmGetScratchBuffer(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo,
                                                   PRE_SUBTASK_TO_SUBTASK, 3 * sizeof(int), nullptr));
    sc[0] = g_extra;
    sc[1] = r1 - r0;
    sc[2] = c1 - c0;
    if (di.deviceType == GPU_CUDA) {
        pmCudaLaunchConf lc(8, 1, 1, 256, 1, 1);
        pmSetCudaLaunchConf(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, lc);
        pmReserveCudaGlobalMem(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo,
                               size_t(r1 - r0) * (c1 - c0) * 4);
    }
    return pmSuccess;
}

pmStatus add_cpu(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const RtConf* conf = static_cast<const RtConf*>(ti.taskConf);
    const int* sc = static_cast<const int*>(
        pmGetScratchBuffer(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, PRE_SUBTASK_TO_SUBTASK, 0, nullptr));
    const int rows = sc[1], cols = sc[2];
    const int* in = static_cast<const int*>(si.memInfo[0].ptr);
    int* out = static_cast<int*>(si.memInfo[1].ptr);
    const int in_ld = si.memInfo[0].visibilityType == SUBSCRIPTION_NATURAL ? conf->ld : cols;
    const int out_ld = si.memInfo[1].visibilityType == SUBSCRIPTION_NATURAL ? conf->ld : cols;
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) out[r * out_ld + c] = in[r * in_ld + c] + conf->add + sc[0];
    return pmSuccess;
}

pmCallbackHandle register_add(bool gpu, const char* key) {
    pmCallbacks cb;
    cb.dataDistribution = add_dd;
    cb.subtask_cpu = add_cpu;
    if (gpu) cb.subtask_gpu_cuda = reinterpret_cast<pmSubtaskCallback_GPU_CUDA>(rt_add_kernel_ptr());
    pmCallbackHandle h = nullptr;
    CHECK(pmRegisterCallbacks(key, cb, &h) == pmSuccess, "register");
    return h;
}

pmMemHandle make_matrix(int seed) {
    pmMemHandle h;
    CHECK(pmCreateMemory2D(kRows, size_t(kCols) * 4, &h) == pmSuccess, "create");
    void* p;
    CHECK(pmGetRawMemPtr(h, &p) == pmSuccess, "raw ptr");
    int* m = static_cast<int*>(p);
    for (int i = 0; i < kRows * kCols; ++i) m[i] = (i * 7919 + seed) % 100003;
    return h;
}

pmTaskHandle submit_add(pmCallbackHandle cb, pmMemHandle in, pmMemHandle out, int add, pmSubscriptionVisibilityType vis,
                        bool cache = true) {
    static RtConf conf;
    conf.add = add;
    conf.ld = kCols;
    pmTaskMem mem[2] = {pmTaskMem(in, READ_ONLY, vis), pmTaskMem(out, WRITE_ONLY, vis)};
    pmTaskDetails td(&conf, sizeof(conf), mem, 2, cb, tiles());
    td.cudaCacheEnabled = cache;
    pmTaskHandle t = nullptr;
    CHECK(pmSubmitTask(td, &t) == pmSuccess, "submit");
    return t;
}

void expect_added(pmMemHandle in_h, pmMemHandle out_h, int add, bool fetch = true) {
    if (fetch) CHECK(pmFetchMemory(out_h) == pmSuccess, "fetch");
    void *ip, *op;
    pmGetRawMemPtr(in_h, &ip);
    pmGetRawMemPtr(out_h, &op);
    const int* in = static_cast<const int*>(ip);
    const int* out = static_cast<const int*>(op);
    for (int i = 0; i < kRows * kCols; ++i)
        CHECK(out[i] == in[i] + add + g_extra, "element %d: got %d expected %d", i, out[i], in[i] + add + g_extra);
}

void test_views(bool gpu, pmSubscriptionVisibilityType vis) {
    pmCallbackHandle cb = register_add(gpu, "ADD");
    pmMemHandle in = make_matrix(1), out;
    CHECK(pmCreateMemory(size_t(kRows) * kCols * 4, &out) == pmSuccess, "create out");
    pmTaskHandle t = submit_add(cb, in, out, 3, vis);
    CHECK(pmWaitForTaskCompletion(t) == pmSuccess, "task failed");
    CHECK(g_sub_status == pmSuccess, "subscription status %d", g_sub_status);
    expect_added(in, out, 3);
    CHECK(pmReleaseTask(t) == pmSuccess, "release");
}

// Three dependent tasks; the intermediates never leave the device.
void test_chain() {
    pmCallbackHandle cb = register_add(true, "ADD");
    pmMemHandle a = make_matrix(2), b, c, d;
    const size_t bytes = size_t(kRows) * kCols * 4;
    pmCreateMemory(bytes, &b);
    pmCreateMemory(bytes, &c);
    pmCreateMemory(bytes, &d);
    pmb_runtime_reset_stats();
    pmTaskHandle t1 = submit_add(cb, a, b, 1, SUBSCRIPTION_OPTIMAL);
    pmTaskHandle t2 = submit_add(cb, b, c, 10, SUBSCRIPTION_OPTIMAL);
    pmTaskHandle t3 = submit_add(cb, c, d, 100, SUBSCRIPTION_OPTIMAL);
    CHECK(pmWaitForTaskCompletion(t3) == pmSuccess && pmWaitForTaskCompletion(t1) == pmSuccess &&
              pmWaitForTaskCompletion(t2) == pmSuccess, "chain failed");
    unsigned long long h2d, d2h, n, batched;
    pmb_runtime_stats(&h2d, &d2h, &n, &batched);
    CHECK(h2d == bytes, "host->device bytes %llu, expected only the first input (%zu)", h2d, bytes);
    CHECK(d2h == 0, "device->host bytes %llu before any fetch", d2h);
    CHECK(n == 3ull * tiles(), "GPU subtasks %llu", n);
    CHECK(pmFetchMemory(d) == pmSuccess, "fetch");
    pmb_runtime_stats(&h2d, &d2h, &n, &batched);
    CHECK(d2h == bytes, "fetch moved %llu bytes", d2h);
    void *ap, *dp;
    pmGetRawMemPtr(a, &ap);
    pmGetRawMemPtr(d, &dp);
    for (int i = 0; i < kRows * kCols; ++i)
        CHECK(static_cast<int*>(dp)[i] == static_cast<int*>(ap)[i] + 111 + 3 * g_extra, "chain element %d", i);
    pmReleaseTask(t1);
    pmReleaseTask(t2);
    pmReleaseTask(t3);
}

// cudaCacheEnabled = false: results reach the host without pmFetchMemory.
void test_write_through() {
    pmCallbackHandle cb = register_add(true, "ADD");
    pmMemHandle in = make_matrix(3), out;
    pmCreateMemory(size_t(kRows) * kCols * 4, &out);
    pmTaskHandle t = submit_add(cb, in, out, 7, SUBSCRIPTION_COMPACT, false);
    CHECK(pmWaitForTaskCompletion(t) == pmSuccess, "task failed");
    expect_added(in, out, 7, false);
    pmReleaseTask(t);
}

// Many tasks in flight at once give the same results as each task alone.
void test_mix() {
    pmCallbackHandle cb = register_add(true, "ADD");
    const int n = 12;
    std::vector<pmMemHandle> ins, outs;
    std::vector<pmTaskHandle> ts;
    for (int k = 0; k < n; ++k) {
        ins.push_back(make_matrix(100 + k));
        pmMemHandle o;
        pmCreateMemory(size_t(kRows) * kCols * 4, &o);
        outs.push_back(o);
    }
    for (int k = 0; k < n; ++k)
        ts.push_back(submit_add(cb, ins[k], outs[k], k, k % 2 ? SUBSCRIPTION_COMPACT : SUBSCRIPTION_NATURAL));
    for (int k = 0; k < n; ++k) {
        CHECK(pmWaitForTaskCompletion(ts[k]) == pmSuccess, "task %d failed", k);
        expect_added(ins[k], outs[k], k);
        pmReleaseTask(ts[k]);
    }
}

pmStatus bad_dd(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    // beyond the end of the address space
    g_sub_status = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION,
                                       pmSubscriptionInfo(1000, 100));
    return si.subtaskId == 1 ? pmUserError : pmSuccess;
}
pmStatus noop_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo) { return pmSuccess; }

void test_errors() {
    pmCallbackHandle h = nullptr;
    std::string longkey(200, 'k');
    CHECK(pmRegisterCallbacks(longkey.c_str(), pmCallbacks(), &h) == pmMaxKeyLengthExceeded, "long key accepted");
    pmCallbacks both;
    both.subtask_gpu_cuda = reinterpret_cast<pmSubtaskCallback_GPU_CUDA>(rt_add_kernel_ptr());
    both.subtask_gpu_custom = reinterpret_cast<pmSubtaskCallback_GPU_Custom>(&noop_cpu);
    CHECK(pmRegisterCallbacks("BOTH", both, &h) == pmInvalidCallbacks, "two GPU callbacks accepted");
    pmCallbacks cb(bad_dd, noop_cpu, (pmSubtaskCallback_GPU_CUDA) nullptr);
    CHECK(pmRegisterCallbacks("BAD", cb, &h) == pmSuccess, "register");
    CHECK(pmRegisterCallbacks("BAD", cb, &h) == pmInvalidKey, "duplicate key accepted");
    pmMemHandle m;
    pmCreateMemory(1024, &m);
    pmTaskMem mem[1] = {pmTaskMem(m, READ_ONLY)};
    pmTaskDetails td(nullptr, 0, mem, 1, h, 2);
    pmTaskHandle t;
    CHECK(pmSubmitTask(td, &t) == pmSuccess, "submit");
    CHECK(pmWaitForTaskCompletion(t) == pmUserError, "data-distribution error not propagated");
    CHECK(g_sub_status == pmInvalidOffset, "out-of-range subscription gave %d", g_sub_status);
    pmReleaseTask(t);
    pmTaskDetails bad = td;
    bad.callbackHandle = reinterpret_cast<pmCallbackHandle>(0x1234);
    CHECK(pmSubmitTask(bad, &t) == pmInvalidCallbacks, "bad callback handle accepted");
    pmRawMemPtr p;
    CHECK(pmGetRawMemPtr(reinterpret_cast<pmMemHandle>(0x1234), &p) == pmUnrecognizedMemory, "bad memory handle");
    CHECK(pmFetchMemoryRange(m, 1000, 100) == pmInvalidOffset, "bad fetch range");
    CHECK(pmReleaseMemory(m) == pmSuccess, "release memory");
    CHECK(pmReleaseMemory(m) == pmUnrecognizedMemory, "double release accepted");
}

pmStatus sleepy_cpu(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo) {
    std::this_thread::sleep_for(std::chrono::milliseconds(1500));
    return pmSuccess;
}
pmStatus empty_dd(pmTaskInfo, pmDeviceInfo, pmSubtaskInfo) { return pmSuccess; }

// A task that outlives its timeout: the wait returns early with an error.
void test_timeout() {
    pmCallbacks cb(empty_dd, sleepy_cpu, (pmSubtaskCallback_GPU_CUDA) nullptr);
    pmCallbackHandle h;
    CHECK(pmRegisterCallbacks("SLEEPY", cb, &h) == pmSuccess, "register");
    pmTaskDetails td(nullptr, 0, nullptr, 0, h, 64);
    td.timeOutInSecs = 1;
    pmTaskHandle t;
    const auto t0 = std::chrono::steady_clock::now();
    CHECK(pmSubmitTask(td, &t) == pmSuccess, "submit");
    const pmStatus st = pmWaitForTaskCompletion(t);
    const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    CHECK(st == pmStatusUnavailable, "timed-out task returned %d", st);
    CHECK(waited < 1.4, "wait took %.2f s", waited);
    const pmStatus rel = pmReleaseTask(t);  // waits until the running subtasks stop
    CHECK(rel == pmStatusUnavailable, "released task status %d", rel);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::printf("usage: rt_selftest <views_cpu|views_cpu_compact|views_gpu|views_gpu_compact|chain|"
                    "write_through|mix|errors|timeout>\n");
        return 2;
    }
    g_test = argv[1];
    CHECK(pmInitialize() == pmSuccess, "init");
    int ndev = 0;
    pmb_device_count(&ndev);
    const bool gpu_test = g_test.find("gpu") != std::string::npos || g_test == "chain" ||
                          g_test == "write_through" || g_test == "mix";
    if (gpu_test) CHECK(ndev > 0 && pmb_device_supported(0), "no supported GPU");
    if (g_test == "views_cpu") test_views(false, SUBSCRIPTION_NATURAL);
    else if (g_test == "views_cpu_compact") test_views(false, SUBSCRIPTION_COMPACT);
    else if (g_test == "views_gpu") test_views(true, SUBSCRIPTION_NATURAL);
    else if (g_test == "views_gpu_compact") test_views(true, SUBSCRIPTION_COMPACT);
    else if (g_test == "chain") test_chain();
    else if (g_test == "write_through") test_write_through();
    else if (g_test == "mix") test_mix();
    else if (g_test == "errors") test_errors();
    else if (g_test == "timeout") test_timeout();
    else CHECK(false, "unknown test");
    CHECK(pmFinalize() == pmSuccess, "finalize");
    std::printf("PASS %s\n", g_test.c_str());
    return 0;
}
