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
#include <type_traits>
#include <vector>
#include <algorithm>
#include <cstdint>

#include "pmPublicDefinitions.h"
#include "pmPublicUtilities.h"
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

// ---------------------------------------------------------------------------
// Subtask reduction: N subtasks each write a private copy of one output range
// (row s of the input, copied or added), folded with a built-in REDUCE_*
// callback or the app's own.  The expected result is folded here in subtask
// order, so float sums are compared bit for bit.

extern "C" void* rt_row_kernel_ptr();

struct RtRowConf {
    int words, accumulate, type, op;
};

constexpr int kRowSubtasks = 7;
constexpr int kRowWords = 2006;  // 8024 bytes: 2006 ints/floats, 1003 longs/doubles

enum class OutSub { Whole, Inner, Scattered, Mismatched };
OutSub g_out_sub = OutSub::Whole;

pmStatus row_dd(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const RtRowConf* conf = static_cast<const RtRowConf*>(ti.taskConf);
    const size_t row = size_t(conf->words) * 4;
    pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION,
                        pmSubscriptionInfo(si.subtaskId * row, row));
    const pmSubscriptionInfo whole(0, row);
    switch (g_out_sub) {
        case OutSub::Whole:
            pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1,
                                conf->accumulate ? READ_WRITE_SUBSCRIPTION : WRITE_SUBSCRIPTION, whole);
            break;
        case OutSub::Inner:  // reads everything, writes [64, row - 8): folded straight into the mirror
            pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, READ_SUBSCRIPTION, whole);
            pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, WRITE_SUBSCRIPTION,
                                pmSubscriptionInfo(64, row - 72));
            break;
        case OutSub::Scattered:  // reads everything, writes 64 of every 128 bytes
            pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, READ_SUBSCRIPTION, whole);
            pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, WRITE_SUBSCRIPTION,
                                pmScatteredSubscriptionInfo(0, 64, 128, row / 128));
            break;
        case OutSub::Mismatched:  // the last subtask writes a shorter range: the task fails
            pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, WRITE_SUBSCRIPTION,
                                pmSubscriptionInfo(0, si.subtaskId + 1 == kRowSubtasks ? row - 64 : row));
            break;
    }
    if (di.deviceType == GPU_CUDA) {
        pmCudaLaunchConf lc(4, 1, 1, 256, 1, 1);
        pmSetCudaLaunchConf(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, lc);
    }
    // a counter that travels with the reductions: subtask id + 1
    uint64_t* counter = static_cast<uint64_t*>(pmGetScratchBuffer(ti.taskHandle, di.deviceHandle, si.subtaskId,
                                                                  si.splitInfo, REDUCTION_TO_REDUCTION, 8, nullptr));
    *counter = si.subtaskId + 1;
    return pmSuccess;
}

pmStatus row_cpu(pmTaskInfo ti, pmDeviceInfo, pmSubtaskInfo si) {
    const RtRowConf* conf = static_cast<const RtRowConf*>(ti.taskConf);
    const unsigned* in = static_cast<const unsigned*>(si.memInfo[0].ptr);
    unsigned* out = static_cast<unsigned*>(si.memInfo[1].ptr);
    for (int j = 0; j < conf->words; ++j) out[j] = conf->accumulate ? out[j] + in[j] : in[j];
    return pmSuccess;
}

// The app's own callbacks: a = a + 3 b over int32, and one that calls
// pmReduceSubtasks (BITWISE_OR, INTS) itself.
pmStatus axpy3_reduction(pmTaskInfo ti, pmDeviceInfo, pmSubtaskInfo s1, pmDeviceInfo, pmSubtaskInfo s2) {
    const RtRowConf* conf = static_cast<const RtRowConf*>(ti.taskConf);
    int* a = static_cast<int*>(s1.memInfo[1].writePtr);
    const int* b = static_cast<const int*>(s2.memInfo[1].writePtr);
    if (!a || !b || s1.memInfo[1].length != size_t(conf->words) * 4) return pmUserError;
    for (int j = 0; j < conf->words; ++j) a[j] += 3 * b[j];
    uint64_t* ca = static_cast<uint64_t*>(pmGetScratchBuffer(ti.taskHandle, nullptr, s1.subtaskId, s1.splitInfo,
                                                             REDUCTION_TO_REDUCTION, 0, nullptr));
    const uint64_t* cb = static_cast<const uint64_t*>(pmGetScratchBuffer(ti.taskHandle, nullptr, s2.subtaskId,
                                                                         s2.splitInfo, REDUCTION_TO_REDUCTION, 0, nullptr));
    if (!ca || !cb) return pmUserError;
    *ca += *cb;
    return pmSuccess;
}

pmStatus or_reduction(pmTaskInfo ti, pmDeviceInfo d1, pmSubtaskInfo s1, pmDeviceInfo d2, pmSubtaskInfo s2) {
    return pmReduceSubtasks(ti.taskHandle, d1.deviceHandle, s1.subtaskId, s1.splitInfo, d2.deviceHandle, s2.subtaskId,
                            s2.splitInfo, REDUCE_BITWISE_OR, REDUCE_INTS);
}

template <typename T, typename B>
T fold_ref(int op, T a, T b) {
    switch (op) {
        case REDUCE_ADD: return a + b;
        case REDUCE_MIN: return b < a ? b : a;
        case REDUCE_MAX: return a < b ? b : a;
        case REDUCE_PRODUCT: return a * b;
        case REDUCE_LOGICAL_AND: return (a != T(0) && b != T(0)) ? T(1) : T(0);
        case REDUCE_BITWISE_AND: return T(B(a) & B(b));
        case REDUCE_LOGICAL_OR: return (a != T(0) || b != T(0)) ? T(1) : T(0);
        case REDUCE_BITWISE_OR: return T(B(a) | B(b));
        case REDUCE_LOGICAL_XOR: return a != b ? T(1) : T(0);
        default: return T(B(a) ^ B(b));
    }
}

bool g_sparse = false;  // inputs mostly zero (sentinel-compressed copies)

template <typename T>
T row_value(int s, int j, int op) {
    const unsigned h = unsigned(j) * 2654435761u + unsigned(s) * 40503u + 17u;
    if (g_sparse && (h >> 7) % 10 != 0) return T(0);
    if (op == REDUCE_LOGICAL_AND || op == REDUCE_LOGICAL_OR || op == REDUCE_LOGICAL_XOR) return T(h % 3);
    if (op == REDUCE_PRODUCT) return T(1 + h % 3);
    if constexpr (std::is_floating_point<T>::value)
        return (op == REDUCE_BITWISE_AND || op == REDUCE_BITWISE_OR || op == REDUCE_BITWISE_XOR)
                   ? T(h % 100000u)
                   : T(int(h % 20001u) - 10000) / T(7);
    else if constexpr (sizeof(T) == 8)
        return T((uint64_t(h) << 29) ^ (uint64_t(h) * 0x9E3779B97F4A7C15ull));
    else
        return T(int(h % 200001u) - 100000);
}

// One task: returns its status; on success compares the output with the fold.
template <typename T, typename B>
void reduce_case(bool gpu, int op, int type, pmDataReductionCallback custom, int custom_kind, int accumulate,
                 OutSub sub, int words = kRowWords) {
    const int n = words * 4 / int(sizeof(T));
    pmCallbacks cb;
    cb.dataDistribution = row_dd;
    cb.subtask_cpu = row_cpu;
    if (gpu) cb.subtask_gpu_cuda = reinterpret_cast<pmSubtaskCallback_GPU_CUDA>(rt_row_kernel_ptr());
    cb.dataReduction = custom ? custom : pmGetSubtaskReductionCallbackImpl(pmReductionOpType(op), pmReductionDataType(type));
    CHECK(cb.dataReduction, "no reduction callback for op %d type %d", op, type);
    char key[32];
    std::snprintf(key, sizeof(key), "ROW_%d_%d_%d_%d", op, type, custom_kind, int(sub));
    pmCallbackHandle h;
    CHECK(pmRegisterCallbacks(key, cb, &h) == pmSuccess, "register");

    pmMemHandle in, out;
    CHECK(pmCreateMemory(size_t(kRowSubtasks) * words * 4, &in) == pmSuccess, "create in");
    CHECK(pmCreateMemory(size_t(words) * 4, &out) == pmSuccess, "create out");
    void *ip, *op_;
    pmGetRawMemPtr(in, &ip);
    pmGetRawMemPtr(out, &op_);
    T* inp = static_cast<T*>(ip);
    T* outp = static_cast<T*>(op_);
    for (int s = 0; s < kRowSubtasks; ++s)
        for (int j = 0; j < n; ++j) inp[size_t(s) * n + j] = row_value<T>(s, j, op);
    std::vector<T> init(n);
    for (int j = 0; j < n; ++j) init[j] = outp[j] = row_value<T>(100, j, op);

    static RtRowConf conf;
    conf = RtRowConf{words, accumulate, type, op};
    g_out_sub = sub;
    const bool reads_out = accumulate || sub == OutSub::Inner || sub == OutSub::Scattered;
    pmTaskMem mem[2] = {pmTaskMem(in, READ_ONLY, SUBSCRIPTION_NATURAL),
                        pmTaskMem(out, reads_out ? READ_WRITE : WRITE_ONLY, SUBSCRIPTION_NATURAL)};
    pmTaskDetails td(&conf, sizeof(conf), mem, 2, h, kRowSubtasks);
    pmTaskHandle t;
    CHECK(pmSubmitTask(td, &t) == pmSuccess, "submit");
    const pmStatus st = pmWaitForTaskCompletion(t);
    if (sub == OutSub::Mismatched) {
        CHECK(st == pmInvalidIndex, "mismatched subscriptions gave status %d", st);
    } else {
        CHECK(st == pmSuccess, "task failed (op %d type %d custom %d sub %d): %d", op, type, custom_kind, int(sub), st);
        CHECK(pmFetchMemory(out) == pmSuccess, "fetch");
        // the subtasks' copies (int32 words when accumulating), folded in order
        std::vector<T> expect(n);
        for (int j = 0; j < n; ++j) {
            T acc{};
            for (int s = 0; s < kRowSubtasks; ++s) {
                T v = inp[size_t(s) * n + j];
                if (accumulate) v = T(int(init[j]) + int(v));
                if (s == 0) acc = v;
                else if (custom_kind == 1) acc = T(int(acc) + 3 * int(v));
                else if (custom_kind == 2) acc = T(int(acc) | int(v));
                else acc = fold_ref<T, B>(op, acc, v);
            }
            const size_t byte = size_t(j) * sizeof(T);
            bool written = true;
            if (sub == OutSub::Inner) written = byte >= 64 && byte < size_t(words) * 4 - 8;
            if (sub == OutSub::Scattered) written = byte % 128 < 64 && byte / 128 < size_t(words) * 4 / 128;
            expect[j] = written ? acc : init[j];
        }
        CHECK(std::memcmp(expect.data(), outp, size_t(n) * sizeof(T)) == 0,
              "op %d type %d custom %d sub %d: first mismatch at %d", op, type, custom_kind, int(sub),
              int(std::mismatch(expect.begin(), expect.end(), outp,
                                [](T a, T b) { return std::memcmp(&a, &b, sizeof(T)) == 0; }).first - expect.begin()));
    }
    if (sub != OutSub::Mismatched) {
        // the REDUCTION_TO_REDUCTION buffer of the subtask all others were folded into: the app's
        // callback summed the counters; the built-in folds leave subtask 0's (1)
        const uint64_t* last = static_cast<const uint64_t*>(pmGetLastReductionScratchBuffer(t));
        const uint64_t want = custom_kind == 1 ? uint64_t(kRowSubtasks) * (kRowSubtasks + 1) / 2 : 1;
        CHECK(last && *last == want, "last reduction scratch %llu expected %llu",
              last ? (unsigned long long)*last : 0ull, (unsigned long long)want);
    }
    CHECK(pmReleaseTask(t) == st, "release");
    CHECK(pmReleaseMemory(in) == pmSuccess && pmReleaseMemory(out) == pmSuccess, "release memory");
    CHECK(pmReleaseCallbacks(h) == pmSuccess, "release callbacks");
}

void test_reduce(bool gpu) {
    CHECK(pmGetSubtaskReductionCallbackImpl(MAX_REDUCTION_OP_TYPES, REDUCE_INTS) == nullptr, "out-of-range op");
    CHECK(pmGetSubtaskReductionCallbackImpl(REDUCE_ADD, MAX_REDUCTION_DATA_TYPES) == nullptr, "out-of-range type");
    // every operation on every data type, whole-range writes
    for (int op = 0; op < MAX_REDUCTION_OP_TYPES; ++op) {
        reduce_case<int32_t, int32_t>(gpu, op, REDUCE_INTS, nullptr, 0, 0, OutSub::Whole);
        reduce_case<uint32_t, uint32_t>(gpu, op, REDUCE_UNSIGNED_INTS, nullptr, 0, 0, OutSub::Whole);
        reduce_case<int64_t, int64_t>(gpu, op, REDUCE_LONGS, nullptr, 0, 0, OutSub::Whole);
        reduce_case<uint64_t, uint64_t>(gpu, op, REDUCE_UNSIGNED_LONGS, nullptr, 0, 0, OutSub::Whole);
        reduce_case<float, uint32_t>(gpu, op, REDUCE_FLOATS, nullptr, 0, 0, OutSub::Whole);
        reduce_case<double, uint64_t>(gpu, op, REDUCE_DOUBLES, nullptr, 0, 0, OutSub::Whole);
    }
    // copies that start from the address space's bytes (READ_WRITE)
    reduce_case<int32_t, int32_t>(gpu, REDUCE_ADD, REDUCE_INTS, nullptr, 0, 1, OutSub::Whole);
    // partial writes: contiguous (folded into the mirror) and scattered
    reduce_case<float, uint32_t>(gpu, REDUCE_ADD, REDUCE_FLOATS, nullptr, 0, 0, OutSub::Inner);
    reduce_case<double, uint64_t>(gpu, REDUCE_MAX, REDUCE_DOUBLES, nullptr, 0, 0, OutSub::Scattered);
    // the app's own callbacks, run on the host
    reduce_case<int32_t, int32_t>(gpu, REDUCE_ADD, REDUCE_INTS, axpy3_reduction, 1, 0, OutSub::Whole);
    reduce_case<int32_t, int32_t>(gpu, REDUCE_BITWISE_OR, REDUCE_INTS, or_reduction, 2, 0, OutSub::Whole);
    reduce_case<int32_t, int32_t>(gpu, REDUCE_ADD, REDUCE_INTS, axpy3_reduction, 1, 0, OutSub::Scattered);
    // a 4 MiB copy per subtask: the host fold splits it over the cores
    reduce_case<float, uint32_t>(gpu, REDUCE_ADD, REDUCE_FLOATS, nullptr, 0, 0, OutSub::Whole, 1 << 20);
    // subtasks subscribing different ranges: the task fails before it runs
    reduce_case<int32_t, int32_t>(gpu, REDUCE_ADD, REDUCE_INTS, nullptr, 0, 0, OutSub::Mismatched);
}

// Sentinel-compressed copies: the app's own reduction callback on GPU
// subtasks whose copies are ~90 % zero words; with the threshold lowered to
// 0 every copy goes to the host compressed, and the folds still match.
extern "C" void pmb_runtime_sentinel_stats(unsigned long long* copies, unsigned long long* bytes);

void test_sentinel() {
    g_sparse = true;
    unsigned long long c0 = 0, b0 = 0, c1 = 0, b1 = 0;
    pmb_runtime_sentinel_stats(&c0, &b0);
    reduce_case<int32_t, int32_t>(true, REDUCE_ADD, REDUCE_INTS, axpy3_reduction, 1, 0, OutSub::Whole);
    reduce_case<int32_t, int32_t>(true, REDUCE_BITWISE_OR, REDUCE_INTS, or_reduction, 2, 0, OutSub::Whole, 1 << 20);
    pmb_runtime_sentinel_stats(&c1, &b1);
    CHECK(c1 - c0 == 2 * kRowSubtasks, "compressed copies: %llu", c1 - c0);
    CHECK(b1 - b0 < (size_t(kRowWords) + (size_t(1) << 20)) * 4 * kRowSubtasks / 4, "compressed bytes %llu", b1 - b0);
    // dense copies stay uncompressed
    g_sparse = false;
    reduce_case<int32_t, int32_t>(true, REDUCE_ADD, REDUCE_INTS, axpy3_reduction, 1, 0, OutSub::Whole);
    unsigned long long c2 = 0;
    pmb_runtime_sentinel_stats(&c2, nullptr);
    CHECK(c2 == c1, "a dense copy was compressed");
}

// ---------------------------------------------------------------------------
// Ordered redistribution: each subtask groups its chunk of keys by bucket and
// its redistribution callback names each bucket's range with order
// subtasks * bucket + subtask, as the reference radixSort does
// (radixSort.cpp:150-162); the address space then holds all keys stably
// grouped by bucket.

extern "C" void* rt_bucket_kernel_ptr();

constexpr int kBuckets = 5, kChunk = 1000, kKeys = 8500;
pmStatus g_redist_bad = pmSuccess;  // status of a deliberately out-of-range pmRedistributeData

int chunk_len(unsigned long id) { return std::min(kChunk, kKeys - int(id) * kChunk); }

pmStatus bucket_dd(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const pmSubscriptionInfo s(si.subtaskId * kChunk * 4, size_t(chunk_len(si.subtaskId)) * 4);
    pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION, s);
    pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, WRITE_SUBSCRIPTION, s);
    pmGetScratchBuffer(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, SUBTASK_TO_POST_SUBTASK,
                       kBuckets * sizeof(int), nullptr);
    if (di.deviceType == GPU_CUDA) {
        pmCudaLaunchConf lc(1, 1, 1, 32, 1, 1);
        pmSetCudaLaunchConf(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, lc);
    }
    return pmSuccess;
}

pmStatus bucket_cpu(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const int* in = static_cast<const int*>(si.memInfo[0].ptr);
    int* out = static_cast<int*>(si.memInfo[1].ptr);
    int* bins = static_cast<int*>(pmGetScratchBuffer(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo,
                                                     SUBTASK_TO_POST_SUBTASK, 0, nullptr));
    const int n = int(si.memInfo[0].length / 4);
    for (int b = 0; b < kBuckets; ++b) bins[b] = 0;
    for (int i = 0; i < n; ++i) bins[in[i] % kBuckets]++;
    int pos = 0;
    for (int b = 0; b < kBuckets; ++b)
        for (int i = 0; i < n; ++i)
            if (in[i] % kBuckets == b) out[pos++] = in[i];
    return pmSuccess;
}

pmStatus bucket_redistribution(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const int* bins = static_cast<const int*>(pmGetScratchBuffer(ti.taskHandle, di.deviceHandle, si.subtaskId,
                                                                 si.splitInfo, SUBTASK_TO_POST_SUBTASK, 0, nullptr));
    if (!bins) return pmUserError;
    size_t off = 0;
    for (int b = 0; b < kBuckets; ++b) {
        const pmStatus st = pmRedistributeData(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, off,
                                               size_t(bins[b]) * 4, uint(ti.subtaskCount * b + si.subtaskId));
        if (st != pmSuccess) return st;
        off += size_t(bins[b]) * 4;
    }
    if (si.subtaskId == 0)  // a range past the end of the address space is refused
        g_redist_bad = pmRedistributeData(ti.taskHandle, di.deviceHandle, 0, si.splitInfo, 1, size_t(kKeys) * 4, 4, 0);
    return pmSuccess;
}

// Each subtask names its chunk as two halves with orders 2 id and 2 id + 1:
// the address space keeps its bytes (ranges that continue one another are
// moved as one copy).
pmStatus halves_redistribution(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const size_t bytes = size_t(chunk_len(si.subtaskId)) * 4, half = bytes / 8 * 4;
    pmStatus st = pmRedistributeData(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, 0, half,
                                     uint(2 * si.subtaskId));
    if (st == pmSuccess)
        st = pmRedistributeData(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, half, bytes - half,
                                uint(2 * si.subtaskId + 1));
    return st;
}

void test_redistribute_halves(bool gpu) {
    pmCallbacks cb;
    cb.dataDistribution = bucket_dd;
    cb.subtask_cpu = bucket_cpu;
    if (gpu) cb.subtask_gpu_cuda = reinterpret_cast<pmSubtaskCallback_GPU_CUDA>(rt_bucket_kernel_ptr());
    cb.dataRedistribution = halves_redistribution;
    pmCallbackHandle h;
    CHECK(pmRegisterCallbacks("HALVES", cb, &h) == pmSuccess, "register");
    pmMemHandle in, out;
    CHECK(pmCreateMemory(size_t(kKeys) * 4, &in) == pmSuccess && pmCreateMemory(size_t(kKeys) * 4, &out) == pmSuccess,
          "create");
    void *ip, *op;
    pmGetRawMemPtr(in, &ip);
    int* keys = static_cast<int*>(ip);
    for (int i = 0; i < kKeys; ++i) keys[i] = int((unsigned(i) * 40503u + 7u) % 100000u);
    static int buckets = kBuckets;
    pmTaskMem mem[2] = {pmTaskMem(in, READ_ONLY, SUBSCRIPTION_NATURAL), pmTaskMem(out, WRITE_ONLY, SUBSCRIPTION_NATURAL)};
    const unsigned long nsub = (kKeys + kChunk - 1) / kChunk;
    pmTaskDetails td(&buckets, sizeof(buckets), mem, 2, h, nsub);
    pmTaskHandle t;
    CHECK(pmSubmitTask(td, &t) == pmSuccess, "submit");
    CHECK(pmWaitForTaskCompletion(t) == pmSuccess, "task failed");
    // each chunk stays where it is, grouped by bucket inside the chunk
    std::vector<int> expect;
    for (unsigned long sub = 0; sub < nsub; ++sub)
        for (int b = 0; b < kBuckets; ++b)
            for (int i = int(sub) * kChunk; i < int(sub) * kChunk + chunk_len(sub); ++i)
                if (keys[i] % kBuckets == b) expect.push_back(keys[i]);
    CHECK(pmFetchMemory(out) == pmSuccess, "fetch");
    pmGetRawMemPtr(out, &op);
    CHECK(std::memcmp(expect.data(), op, size_t(kKeys) * 4) == 0, "halves redistribution moved bytes");
    ulong count = 0;
    const pmRedistributionMetadata* md = pmGetRedistributionMetadata(t, 1, &count);
    CHECK(md && count == 2 * nsub, "metadata count %lu", count);
    for (unsigned long sub = 0; sub < nsub; ++sub) {
        const uint bytes = uint(chunk_len(sub)) * 4, half = bytes / 8 * 4;
        CHECK(md[2 * sub].order == 2 * sub && md[2 * sub].count == half && md[2 * sub + 1].count == bytes - half,
              "metadata of subtask %lu", sub);
    }
    CHECK(pmReleaseTask(t) == pmSuccess, "release");
    CHECK(pmReleaseMemory(in) == pmSuccess && pmReleaseMemory(out) == pmSuccess, "release memory");
}

void test_redistribute(bool gpu) {
    pmCallbacks cb;
    cb.dataDistribution = bucket_dd;
    cb.subtask_cpu = bucket_cpu;
    if (gpu) cb.subtask_gpu_cuda = reinterpret_cast<pmSubtaskCallback_GPU_CUDA>(rt_bucket_kernel_ptr());
    cb.dataRedistribution = bucket_redistribution;
    pmCallbackHandle h;
    CHECK(pmRegisterCallbacks("BUCKETS", cb, &h) == pmSuccess, "register");
    pmMemHandle in, out;
    CHECK(pmCreateMemory(size_t(kKeys) * 4, &in) == pmSuccess && pmCreateMemory(size_t(kKeys) * 4, &out) == pmSuccess,
          "create");
    void *ip, *op;
    pmGetRawMemPtr(in, &ip);
    int* keys = static_cast<int*>(ip);
    for (int i = 0; i < kKeys; ++i) keys[i] = int((unsigned(i) * 2654435761u) % 100000u);
    static int buckets = kBuckets;
    pmTaskMem mem[2] = {pmTaskMem(in, READ_ONLY, SUBSCRIPTION_NATURAL), pmTaskMem(out, WRITE_ONLY, SUBSCRIPTION_NATURAL)};
    const unsigned long nsub = (kKeys + kChunk - 1) / kChunk;
    pmTaskDetails td(&buckets, sizeof(buckets), mem, 2, h, nsub);
    pmTaskHandle t;
    CHECK(pmSubmitTask(td, &t) == pmSuccess, "submit");
    CHECK(pmWaitForTaskCompletion(t) == pmSuccess, "task failed");
    CHECK(g_redist_bad == pmInvalidIndex, "out-of-range redistribution returned %d", g_redist_bad);
    pmSplitInfo split;
    CHECK(pmRedistributeData(t, nullptr, 0, split, 1, 0, 4, 0) == pmInvalidCommand,
          "redistribution accepted after the task");
    // expected: keys stably grouped by bucket over the whole array; metadata per (bucket, subtask)
    std::vector<int> expect;
    std::vector<std::pair<uint, uint>> meta;
    for (int b = 0; b < kBuckets; ++b)
        for (unsigned long s = 0; s < nsub; ++s) {
            uint bytes = 0;
            for (int i = int(s) * kChunk; i < int(s) * kChunk + chunk_len(s); ++i)
                if (keys[i] % kBuckets == b) {
                    expect.push_back(keys[i]);
                    bytes += 4;
                }
            if (bytes) meta.emplace_back(uint(nsub * b + s), bytes);
        }
    CHECK(pmFetchMemory(out) == pmSuccess, "fetch");
    pmGetRawMemPtr(out, &op);
    CHECK(int(expect.size()) == kKeys && std::memcmp(expect.data(), op, size_t(kKeys) * 4) == 0,
          "redistributed keys differ");
    ulong count = 0;
    const pmRedistributionMetadata* md = pmGetRedistributionMetadata(t, 1, &count);
    CHECK(md && count == meta.size(), "metadata count %lu expected %zu", count, meta.size());
    for (size_t k = 0; k < meta.size(); ++k)
        CHECK(md[k].order == meta[k].first && md[k].count == meta[k].second, "metadata %zu: (%u, %u) expected (%u, %u)",
              k, md[k].order, md[k].count, meta[k].first, meta[k].second);
    ulong none = 7;
    CHECK(pmGetRedistributionMetadata(t, 0, &none) == nullptr && none == 0, "metadata of an address space not redistributed");
    CHECK(pmReleaseTask(t) == pmSuccess, "release");
    CHECK(pmReleaseMemory(in) == pmSuccess && pmReleaseMemory(out) == pmSuccess, "release memory");
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::printf("usage: rt_selftest <views_cpu|views_cpu_compact|views_gpu|views_gpu_compact|chain|"
                    "write_through|mix|errors|timeout|reduce_cpu|reduce_gpu|sentinel_gpu|redistribute_cpu|redistribute_gpu>\n");
        return 2;
    }
    g_test = argv[1];
    if (g_test == "sentinel_gpu") setenv("PMB_SENTINEL_THRESHOLD_BYTES", "0", 1);
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
    else if (g_test == "reduce_cpu") test_reduce(false);
    else if (g_test == "reduce_gpu") test_reduce(true);
    else if (g_test == "sentinel_gpu") test_sentinel();
    else if (g_test == "redistribute_cpu") {
        test_redistribute(false);
        test_redistribute_halves(false);
    } else if (g_test == "redistribute_gpu") {
        test_redistribute(true);
        test_redistribute_halves(true);
    }
    else CHECK(false, "unknown test");
    CHECK(pmFinalize() == pmSuccess, "finalize");
    std::printf("PASS %s\n", g_test.c_str());
    return 0;
}
