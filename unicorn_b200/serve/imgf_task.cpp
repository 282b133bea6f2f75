// imageFiltering task over the pm:: API, timed end to end.
//
// This is an app of the pm:: runtime written the way the reference's
// imageFiltering app is (testSuite/imageFiltering/source/code/src/
// imageFiltering.cpp: DoParallelProcess :607-663, parallelImageFilter
// :213-277): the input image lives in a 2-D address space the app fills on the
// host, one task of (W / tile) x (H / tile) subtasks filters it into an output
// address space, and the app fetches the output to the host.  Its data
// distribution restates imageFilterDataDistribution / GetSubtaskSubscription
// (:279-377): subtask k owns output tile (k / tilesPerRow, k % tilesPerRow);
// it reads the tile plus an R-pixel halo clamped to the image from the
// bottom-up input rows and writes the tile of the top-down output.  The GPU
// callback runs the B200 stencil of libpmb.so on the subscription views
// (NATURAL), with a batch hook so the runtime launches groups of subtasks
// together; edge mode clamp (output clamped to [0, 255]) or wrap (the
// reference's signed-char accumulation).
//
// One timed step: the app touches its input on the host (pmGetRawMemPtr, so
// the runtime must stage it to the device again), submits the task, waits for
// it, fetches the output address space (pmFetchMemory) and reads it on the
// host (pmGetRawMemPtr).  With --cache 0 (the default here) the task runs
// with cudaCacheEnabled = false: results are written back during the task.
// Steps run back to back; each step's host wall time is recorded.
//
// Output: one JSON object on stdout.  --dump PREFIX also writes PREFIX.in,
// PREFIX.filter and PREFIX.out (raw bytes) for the tests' oracle check.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pmPublicDefinitions.h"
#include "pmb_capi.h"

using namespace pm;

extern "C" int pmb_runtime_register_batch(void* subtask_gpu_custom, void* batch_fn);
extern "C" void pmb_runtime_stats(unsigned long long* h2d_bytes, unsigned long long* d2h_bytes,
                                  unsigned long long* gpu_subtasks, unsigned long long* batched_launches);
extern "C" void pmb_runtime_reset_stats(void);
extern "C" void pmb_runtime_timers(double* stub_s, double* admit_wait_s, double* pinned_alloc_s,
                                   unsigned long long* pinned_alloc_bytes);
extern "C" double pmb_runtime_callback_seconds(void);

namespace {

constexpr unsigned kIn = 0, kOut = 1;

struct ImgfConf {
    int width, height, tile, radius, mode;
    int8_t filter[PMB_IMGF_MAX_FILTER_DIM * PMB_IMGF_MAX_FILTER_DIM];
};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Output tile of subtask `id` (row-major over tiles), clipped to the image.
void tile_of(const ImgfConf& c, unsigned long id, int* r0, int* r1, int* c0, int* c1) {
    const int per_row = (c.width + c.tile - 1) / c.tile;
    *c0 = static_cast<int>(id % per_row) * c.tile;
    *r0 = static_cast<int>(id / per_row) * c.tile;
    *c1 = std::min(*c0 + c.tile, c.width);
    *r1 = std::min(*r0 + c.tile, c.height);
}

pmStatus imgf_distribution(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const ImgfConf& c = *static_cast<const ImgfConf*>(ti.taskConf);
    int r0, r1, c0, c1;
    tile_of(c, si.subtaskId, &r0, &r1, &c0, &c1);
    const size_t row = 3ull * c.width;
    const int first_row = std::max(r0 - c.radius, 0), last_row = std::min(r1 - 1 + c.radius, c.height - 1);
    const int first_col = std::max(c0 - c.radius, 0), last_col = std::min(c1 - 1 + c.radius, c.width - 1);
    // Input rows are stored bottom-up: image row m is address-space row H-1-m.
    const size_t inv_last = static_cast<size_t>(c.height - 1 - last_row);
    const size_t inv_first = static_cast<size_t>(c.height - 1 - first_row);
    pmStatus st = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, kIn, READ_SUBSCRIPTION,
                                      pmScatteredSubscriptionInfo(inv_last * row + 3ull * first_col,
                                                                  3ull * (last_col - first_col + 1), row,
                                                                  inv_first - inv_last + 1));
    if (st != pmSuccess) return st;
    return pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, kOut, WRITE_SUBSCRIPTION,
                               pmScatteredSubscriptionInfo(static_cast<size_t>(r0) * row + 3ull * c0, 3ull * (c1 - c0),
                                                           row, static_cast<size_t>(r1 - r0)));
}

// Stencil item of one subtask from its NATURAL views: the views start at the
// first subscribed byte (input: bottom-up row H-1-last_row, column first_col).
pmb_imgf_item item_of(const ImgfConf& c, const pmSubtaskInfo& si) {
    int r0, r1, c0, c1;
    tile_of(c, si.subtaskId, &r0, &r1, &c0, &c1);
    const int last_row = std::min(r1 - 1 + c.radius, c.height - 1);
    const int first_col = std::max(c0 - c.radius, 0);
    pmb_imgf_item it;
    it.in = static_cast<const uint8_t*>(si.memInfo[kIn].ptr);
    it.out = static_cast<uint8_t*>(si.memInfo[kOut].ptr);
    it.in_pitch = it.out_pitch = 3LL * c.width;
    it.width = c.width;
    it.height = c.height;
    it.in_row0 = c.height - 1 - last_row;
    it.in_col0 = first_col;
    it.out_row0 = r0;
    it.out_col0 = c0;
    it.r0 = r0;
    it.r1 = r1;
    it.c0 = c0;
    it.c1 = c1;
    return it;
}

pmStatus to_pm(int st) { return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st); }

pmStatus imgf_gpu(pmTaskInfo ti, pmDeviceInfo, pmSubtaskInfo si, void* stream) {
    const ImgfConf& c = *static_cast<const ImgfConf*>(ti.taskConf);
    const pmb_imgf_item it = item_of(c, si);
    return to_pm(pmb_image_filter(&it, 1, c.filter, c.radius, c.mode, stream));
}

pmStatus imgf_gpu_batch(const pmTaskInfo* ti, const pmDeviceInfo*, const pmSubtaskInfo* subtasks, unsigned long count,
                        void* stream) {
    const ImgfConf& c = *static_cast<const ImgfConf*>(ti->taskConf);
    pmb_imgf_item items[PMB_IMGF_MAX_ITEMS];
    for (unsigned long b = 0; b < count; b += PMB_IMGF_MAX_ITEMS) {
        const unsigned long n = std::min<unsigned long>(count - b, PMB_IMGF_MAX_ITEMS);
        for (unsigned long k = 0; k < n; ++k) items[k] = item_of(c, subtasks[b + k]);
        const int st = pmb_image_filter(items, static_cast<int>(n), c.filter, c.radius, c.mode, stream);
        if (st != PMB_SUCCESS) return to_pm(st);
    }
    return pmSuccess;
}

struct Options {
    int width = 8192, height = 8192, tile = 512, radius = 2, mode = PMB_IMGF_CLAMP;
    int steps = 20, warmup = 5, cache = 0;
    uint64_t seed = 3;
    std::string dump;
};

bool parse(int argc, char** argv, Options& o) {
    for (int i = 1; i + 1 < argc; i += 2) {
        const std::string k = argv[i];
        const char* v = argv[i + 1];
        if (k == "--width") o.width = atoi(v);
        else if (k == "--height") o.height = atoi(v);
        else if (k == "--tile") o.tile = atoi(v);
        else if (k == "--radius") o.radius = atoi(v);
        else if (k == "--mode") o.mode = std::string(v) == "wrap" ? PMB_IMGF_WRAP : PMB_IMGF_CLAMP;
        else if (k == "--steps") o.steps = atoi(v);
        else if (k == "--warmup") o.warmup = atoi(v);
        else if (k == "--cache") o.cache = atoi(v);
        else if (k == "--seed") o.seed = strtoull(v, nullptr, 10);
        else if (k == "--dump") o.dump = v;
        else return false;
    }
    return o.width > 0 && o.height > 0 && o.tile > 0 && o.radius >= 1 && o.radius <= 15 && o.steps >= 1;
}

int die(const char* what, pmStatus st) {
    std::fprintf(stderr, "imgf_task: %s failed (%d): %s\n", what, static_cast<int>(st), pmGetLastError());
    return 1;
}

bool write_file(const std::string& path, const void* p, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(p, 1, n, f) == n;
    return std::fclose(f) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    if (!parse(argc, argv, o)) {
        std::fprintf(stderr,
                     "usage: imgf_task [--width W] [--height H] [--tile T] [--radius R] [--mode clamp|wrap] "
                     "[--steps K] [--warmup W] [--cache 0|1] [--seed S] [--dump PREFIX]\n");
        return 2;
    }
    pmStatus st = pmInitialize();
    if (st != pmSuccess) return die("pmInitialize", st);

    ImgfConf conf;
    std::memset(&conf, 0, sizeof(conf));
    conf.width = o.width;
    conf.height = o.height;
    conf.tile = o.tile;
    conf.radius = o.radius;
    conf.mode = o.mode;
    uint64_t s = o.seed;
    const int fd = 2 * o.radius + 1;
    for (int r = 0; r < fd; ++r)
        for (int c = 0; c < fd; ++c)
            conf.filter[r * PMB_IMGF_MAX_FILTER_DIM + c] = static_cast<int8_t>(static_cast<int>(splitmix(s) % 9) - 4);

    const size_t bytes = 3ull * o.width * o.height;
    pmMemHandle in = nullptr, out = nullptr;
    if ((st = pmCreateMemory2D(o.height, 3ull * o.width, &in)) != pmSuccess) return die("pmCreateMemory2D", st);
    if ((st = pmCreateMemory2D(o.height, 3ull * o.width, &out)) != pmSuccess) return die("pmCreateMemory2D", st);
    pmRawMemPtr raw = nullptr;
    if ((st = pmGetRawMemPtr(in, &raw)) != pmSuccess) return die("pmGetRawMemPtr", st);
    {
        uint64_t* w = static_cast<uint64_t*>(raw);
        for (size_t i = 0; i < bytes / 8; ++i) w[i] = splitmix(s);
        for (size_t i = bytes / 8 * 8; i < bytes; ++i) static_cast<uint8_t*>(raw)[i] = static_cast<uint8_t>(splitmix(s));
    }

    pmCallbacks cb;
    cb.dataDistribution = imgf_distribution;
    cb.subtask_gpu_custom = imgf_gpu;
    pmCallbackHandle handle = nullptr;
    if ((st = pmRegisterCallbacks("imgf_b200_e2e", cb, &handle)) != pmSuccess) return die("pmRegisterCallbacks", st);
    pmb_runtime_register_batch(reinterpret_cast<void*>(&imgf_gpu), reinterpret_cast<void*>(&imgf_gpu_batch));

    const unsigned long subtasks = static_cast<unsigned long>((o.width + o.tile - 1) / o.tile) *
                                   static_cast<unsigned long>((o.height + o.tile - 1) / o.tile);
    pmTaskMem mem[2];
    mem[kIn] = pmTaskMem(in, READ_ONLY, SUBSCRIPTION_OPTIMAL);
    mem[kOut] = pmTaskMem(out, WRITE_ONLY, SUBSCRIPTION_OPTIMAL);

    auto step = [&](double* ms) -> pmStatus {
        const double t0 = now_s();
        pmRawMemPtr p = nullptr;
        pmStatus e = pmGetRawMemPtr(in, &p);  // the app touches its input on the host
        if (e != pmSuccess) return e;
        pmTaskDetails td(&conf, sizeof(conf), mem, 2, handle, subtasks);
        td.policy = SLOW_START;
        td.cudaCacheEnabled = o.cache != 0;
        pmTaskHandle task = nullptr;
        if ((e = pmSubmitTask(td, &task)) != pmSuccess) return e;
        e = pmWaitForTaskCompletion(task);
        const pmStatus rel = pmReleaseTask(task);
        if (e != pmSuccess) return e;
        if (rel != pmSuccess) return rel;
        if ((e = pmFetchMemory(out)) != pmSuccess) return e;
        if ((e = pmGetRawMemPtr(out, &p)) != pmSuccess) return e;
        volatile uint8_t sink = static_cast<const uint8_t*>(p)[bytes - 1];  // the result is in host memory
        (void)sink;
        *ms = (now_s() - t0) * 1e3;
        return pmSuccess;
    };

    double ms = 0;
    for (int w = 0; w < o.warmup; ++w)
        if ((st = step(&ms)) != pmSuccess) return die("warm-up task", st);
    pmb_runtime_reset_stats();
    std::vector<double> times;
    const double t_all = now_s();
    for (int k = 0; k < o.steps; ++k) {
        if ((st = step(&ms)) != pmSuccess) return die("task", st);
        times.push_back(ms);
    }
    const double total_ms = (now_s() - t_all) * 1e3;
    unsigned long long h2d = 0, d2h = 0, gsub = 0, batched = 0;
    pmb_runtime_stats(&h2d, &d2h, &gsub, &batched);
    double stub_s = 0, admit_s = 0, pin_s = 0;
    unsigned long long pin_b = 0;
    pmb_runtime_timers(&stub_s, &admit_s, &pin_s, &pin_b);
    const double cb_s = pmb_runtime_callback_seconds();

    if (!o.dump.empty()) {
        pmRawMemPtr pi = nullptr, po = nullptr;
        pmGetRawMemPtr(in, &pi);
        pmGetRawMemPtr(out, &po);
        std::vector<int8_t> f(conf.filter, conf.filter + sizeof(conf.filter));
        if (!write_file(o.dump + ".in", pi, bytes) || !write_file(o.dump + ".out", po, bytes) ||
            !write_file(o.dump + ".filter", f.data(), f.size())) {
            std::fprintf(stderr, "imgf_task: cannot write %s.*\n", o.dump.c_str());
            return 1;
        }
    }
    pmReleaseMemory(in);
    pmReleaseMemory(out);
    pmReleaseCallbacks(handle);
    pmFinalize();

    std::vector<double> sorted = times;
    std::sort(sorted.begin(), sorted.end());
    const double mean = total_ms / o.steps;
    const double alg = 2.0 * static_cast<double>(bytes);
    std::printf(
        "{\"workload\": \"imageFiltering task over the pm:: API: %dx%d RGB u8, %dx%d filter, %s, %lu subtasks of "
        "%dx%d\", \"steps\": %d, \"warmup\": %d, \"cuda_cache\": %d, \"ms_per_step\": %.4f, \"ms_p50\": %.4f, "
        "\"ms_min\": %.4f, \"gbs\": %.2f, \"h2d_bytes_per_step\": %.0f, \"d2h_bytes_per_step\": %.0f, "
        "\"batched_launches_per_task\": %.2f, \"stub_ms_per_task\": %.4f, \"callback_ms_per_task\": %.4f}\n",
        o.width, o.height, fd, fd, o.mode == PMB_IMGF_CLAMP ? "clamp" : "wrap", subtasks, o.tile, o.tile, o.steps,
        o.warmup, o.cache, mean, sorted[sorted.size() / 2], sorted.front(), alg / (mean * 1e-3) / 1e9,
        static_cast<double>(h2d) / o.steps, static_cast<double>(d2h) / o.steps,
        static_cast<double>(batched) / o.steps, stub_s * 1e3 / o.steps, cb_s * 1e3 / o.steps);
    return 0;
}
