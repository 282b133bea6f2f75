// prefixSum and radixSort as pm:: API apps on the B200 runtime.
//
// The reference apps (testSuite/prefixSum/source/code/src/prefixSum.cpp,
// testSuite/radixSort/source/code/src/radixSort.cpp) use an older pm:: API and
// do not compile against the current one; this program runs their task
// structure on the current API with the B200 GPU callbacks of
// libpmb_app_prefixSum.so / libpmb_app_radixSort.so:
//
//   prefix: task 1 scans each subtask's slice (uint32 in, uint64 sums out;
//           scan state in reserved device memory); the app reads each slice's
//           last sum (pmFetchMemoryRange) and scans them on the host into an
//           auxiliary address space (PopulateAuxMem, prefixSum.cpp:191-214);
//           task 2 adds total i to slice i + 1 (ParallelAddAuxArray, :216-243).
//   sort:   one task per LSD round (ParallelSort, radixSort.cpp:177-201):
//           every subtask sorts its slice stably on the round's digit and
//           keeps its digit counts in a SUBTASK_TO_POST_SUBTASK scratch buffer;
//           the redistribution callback orders the keys digit-major,
//           subtask-minor; the rounds alternate between two address spaces.
//
// Inputs are uniform uint32 keys from a seed.  Each step is the whole flow,
// timed on the host clock; the result is checked after the timed steps
// (prefix: consecutive differences equal the keys; sort: non-decreasing and a
// permutation of the keys).  --dump PREFIX writes PREFIX.in / PREFIX.out for
// the tests' oracle check.  Output: one JSON object on stdout.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pmPublicDefinitions.h"
#include "pmb_capi.h"
#include "prefixSum_b200.h"
#include "radixSort_b200.h"

using namespace pm;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Options {
    std::string mode = "prefix";
    uint64_t n = uint64_t(1) << 28;
    uint64_t per = uint64_t(1) << 22;
    int bits = 8, steps = 3, warmup = 1;
    uint64_t seed = 2;
    std::string dump;
};

bool parse(int argc, char** argv, Options& o) {
    if (argc < 2) return false;
    o.mode = argv[1];
    for (int i = 2; i + 1 < argc; i += 2) {
        const std::string k = argv[i];
        const char* v = argv[i + 1];
        if (k == "--n") o.n = strtoull(v, nullptr, 10);
        else if (k == "--per") o.per = strtoull(v, nullptr, 10);
        else if (k == "--bits") o.bits = atoi(v);
        else if (k == "--steps") o.steps = atoi(v);
        else if (k == "--warmup") o.warmup = atoi(v);
        else if (k == "--seed") o.seed = strtoull(v, nullptr, 10);
        else if (k == "--dump") o.dump = v;
        else return false;
    }
    return (o.mode == "prefix" || o.mode == "sort") && o.n >= 1 && o.per >= 1 && o.per % 4 == 0 &&
           (o.bits == 4 || o.bits == 8) && o.steps >= 1 && o.n < (uint64_t(1) << 30);
}

int die(const char* what, pmStatus st) {
    std::fprintf(stderr, "scan_sort_tasks: %s failed (%d): %s\n", what, static_cast<int>(st), pmGetLastError());
    return 1;
}

uint64_t slice_len(uint64_t n, uint64_t per, unsigned long id) { return std::min(per, n - id * per); }

// ---- prefix sum: the app's data distributions ------------------------------

pmStatus scan_dd(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const prefixSum::prefixSumTaskConf* c = static_cast<const prefixSum::prefixSumTaskConf*>(ti.taskConf);
    const uint64_t len = slice_len(c->arrayLen, c->elemsPerSubtask, si.subtaskId);
    const uint64_t first = si.subtaskId * c->elemsPerSubtask;
    pmStatus st = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION,
                                      pmSubscriptionInfo(first * 4, len * 4));
    if (st == pmSuccess)
        st = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, WRITE_SUBSCRIPTION,
                                 pmSubscriptionInfo(first * 8, len * 8));
    if (st == pmSuccess && di.deviceType == GPU_CUDA)
        st = pmReserveCudaGlobalMem(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo,
                                    prefixSum::prefixSumReservedBytes(len));
    return st;
}

pmStatus add_dd(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const prefixSum::prefixSumTaskConf* c = static_cast<const prefixSum::prefixSumTaskConf*>(ti.taskConf);
    const uint64_t len = slice_len(c->arrayLen, c->elemsPerSubtask, si.subtaskId + 1);
    pmStatus st = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION,
                                      pmSubscriptionInfo(si.subtaskId * 8, 8));
    if (st == pmSuccess)
        st = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1,
                                 READ_WRITE_SUBSCRIPTION,
                                 pmSubscriptionInfo((si.subtaskId + 1) * c->elemsPerSubtask * 8, len * 8));
    return st;
}

// ---- radix sort: the app's data distribution --------------------------------

pmStatus sort_dd(pmTaskInfo ti, pmDeviceInfo di, pmSubtaskInfo si) {
    const radixSort::radixSortTaskConf* c = static_cast<const radixSort::radixSortTaskConf*>(ti.taskConf);
    const uint64_t len = slice_len(c->arrayLen, c->elemsPerSubtask, si.subtaskId);
    const pmSubscriptionInfo slice(si.subtaskId * c->elemsPerSubtask * 4, len * 4);
    pmStatus st = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION,
                                      slice);
    if (st == pmSuccess)
        st = pmSubscribeToMemory(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo, 1, WRITE_SUBSCRIPTION,
                                 slice);
    if (st == pmSuccess && !pmGetScratchBuffer(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo,
                                               SUBTASK_TO_POST_SUBTASK, sizeof(uint32_t) << c->bitsPerRound, nullptr))
        st = pmMemoryError;
    if (st == pmSuccess && di.deviceType == GPU_CUDA)
        st = pmReserveCudaGlobalMem(ti.taskHandle, di.deviceHandle, si.subtaskId, si.splitInfo,
                                    radixSort::radixSortReservedBytes(len, c->bitsPerRound));
    return st;
}

pmStatus run_task(pmTaskDetails td) {
    pmTaskHandle t = nullptr;
    pmStatus st = pmSubmitTask(td, &t);
    if (st != pmSuccess) return st;
    st = pmWaitForTaskCompletion(t);
    const pmStatus rel = pmReleaseTask(t);
    return st != pmSuccess ? st : rel;
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
        std::fprintf(stderr, "usage: scan_sort_tasks prefix|sort [--n N] [--per ELEMS_PER_SUBTASK] [--bits 4|8] "
                             "[--steps K] [--warmup W] [--seed S] [--dump PREFIX]\n");
        return 2;
    }
    pmStatus st = pmInitialize();
    if (st != pmSuccess) return die("pmInitialize", st);
    const unsigned long subtasks = static_cast<unsigned long>((o.n + o.per - 1) / o.per);
    std::vector<uint32_t> keys(o.n);
    uint64_t s = o.seed;
    for (auto& k : keys) k = static_cast<uint32_t>(splitmix(s) >> 32);

    pmMemHandle in = nullptr, out = nullptr, aux = nullptr;
    const bool prefix = o.mode == "prefix";
    if ((st = pmCreateMemory(o.n * 4, &in)) != pmSuccess) return die("pmCreateMemory", st);
    if ((st = pmCreateMemory(o.n * (prefix ? 8 : 4), &out)) != pmSuccess) return die("pmCreateMemory", st);
    if (prefix && (st = pmCreateMemory(subtasks * 8, &aux)) != pmSuccess) return die("pmCreateMemory", st);

    pmCallbacks cb1, cb2;
    pmCallbackHandle h1 = nullptr, h2 = nullptr;
    if (prefix) {
        cb1.dataDistribution = scan_dd;
        cb1.subtask_gpu_custom = prefixSum::prefixSum_cudaLaunchFunc;
        cb2.dataDistribution = add_dd;
        cb2.subtask_gpu_custom = prefixSum::elemAdd_cudaLaunchFunc;
        if ((st = pmRegisterCallbacks("PREFIX_SUM", cb1, &h1)) != pmSuccess ||
            (st = pmRegisterCallbacks("ELEM_ADD", cb2, &h2)) != pmSuccess)
            return die("pmRegisterCallbacks", st);
    } else {
        cb1.dataDistribution = sort_dd;
        cb1.subtask_gpu_custom = radixSort::radixSort_cudaLaunchFunc;
        cb1.dataRedistribution = radixSort::radixSortDataRedistribution;
        if ((st = pmRegisterCallbacks("RADIX_SORT", cb1, &h1)) != pmSuccess) return die("pmRegisterCallbacks", st);
    }

    // One step: the input is written on the host, the flow runs, the result
    // is fetched to the host.
    pmMemHandle result = out;
    auto step = [&](double* ms) -> pmStatus {
        const double t0 = now_s();
        pmRawMemPtr p = nullptr;
        pmStatus e = pmGetRawMemPtr(in, &p);
        if (e != pmSuccess) return e;
        std::memcpy(p, keys.data(), o.n * 4);
        if (prefix) {
            prefixSum::prefixSumTaskConf conf{o.n, o.per};
            pmTaskMem mem[2] = {pmTaskMem(in, READ_ONLY, SUBSCRIPTION_NATURAL), pmTaskMem(out, WRITE_ONLY, SUBSCRIPTION_NATURAL)};
            pmTaskDetails td(&conf, sizeof(conf), mem, 2, h1, subtasks);
            if ((e = run_task(td)) != pmSuccess) return e;
            if (subtasks > 1) {
                pmRawMemPtr po = nullptr, pa = nullptr;
                if ((e = pmGetRawMemPtr(aux, &pa)) != pmSuccess) return e;
                uint64_t* a = static_cast<uint64_t*>(pa);
                uint64_t run = 0;
                for (unsigned long i = 0; i < subtasks; ++i) {  // last sum of each slice, scanned
                    const uint64_t last = std::min<uint64_t>((i + 1) * o.per, o.n) - 1;
                    if ((e = pmFetchMemoryRange(out, last * 8, 8)) != pmSuccess) return e;
                    if ((e = pmGetRawMemPtr(out, &po)) != pmSuccess) return e;
                    run += static_cast<const uint64_t*>(po)[last];
                    a[i] = run;
                }
                pmTaskMem mem2[2] = {pmTaskMem(aux, READ_ONLY, SUBSCRIPTION_NATURAL),
                                     pmTaskMem(out, READ_WRITE, SUBSCRIPTION_NATURAL, true)};
                pmTaskDetails td2(&conf, sizeof(conf), mem2, 2, h2, subtasks - 1);
                if ((e = run_task(td2)) != pmSuccess) return e;
            }
            result = out;
        } else {
            pmMemHandle a = in, b = out;
            const int rounds = 32 / o.bits;
            for (int r = 0; r < rounds; ++r) {
                radixSort::radixSortTaskConf conf{o.n, o.per, r, o.bits};
                pmTaskMem mem[2] = {pmTaskMem(a, READ_ONLY, SUBSCRIPTION_NATURAL), pmTaskMem(b, WRITE_ONLY, SUBSCRIPTION_NATURAL)};
                pmTaskDetails td(&conf, sizeof(conf), mem, 2, h1, subtasks);
                if ((e = run_task(td)) != pmSuccess) return e;
                std::swap(a, b);
            }
            result = a;
        }
        if ((e = pmFetchMemory(result)) != pmSuccess) return e;
        pmRawMemPtr pr = nullptr;
        if ((e = pmGetRawMemPtr(result, &pr)) != pmSuccess) return e;
        *ms = (now_s() - t0) * 1e3;
        return pmSuccess;
    };

    double ms = 0;
    for (int w = 0; w < o.warmup; ++w)
        if ((st = step(&ms)) != pmSuccess) return die("warm-up flow", st);
    std::vector<double> times;
    for (int k = 0; k < o.steps; ++k) {
        if ((st = step(&ms)) != pmSuccess) return die("flow", st);
        times.push_back(ms);
    }
    pmRawMemPtr pr = nullptr;
    pmGetRawMemPtr(result, &pr);
    bool ok = true;
    if (prefix) {
        const uint64_t* y = static_cast<const uint64_t*>(pr);
        ok = y[0] == keys[0];
        for (uint64_t i = 1; i < o.n && ok; ++i) ok = y[i] - y[i - 1] == keys[i];
    } else {
        const uint32_t* y = static_cast<const uint32_t*>(pr);
        uint64_t sum_in = 0, sum_out = 0, x_in = 0, x_out = 0;
        for (uint64_t i = 0; i < o.n; ++i) {
            sum_in += keys[i];
            sum_out += y[i];
            x_in ^= keys[i] * 0x9E3779B97F4A7C15ull;
            x_out ^= y[i] * 0x9E3779B97F4A7C15ull;
            if (i && y[i] < y[i - 1]) ok = false;
        }
        ok = ok && sum_in == sum_out && x_in == x_out;
    }
    if (!o.dump.empty()) {
        if (!write_file(o.dump + ".in", keys.data(), o.n * 4) ||
            !write_file(o.dump + ".out", pr, o.n * (prefix ? 8 : 4))) {
            std::fprintf(stderr, "scan_sort_tasks: cannot write %s.*\n", o.dump.c_str());
            return 1;
        }
    }
    pmReleaseMemory(in);
    pmReleaseMemory(out);
    if (aux) pmReleaseMemory(aux);
    pmReleaseCallbacks(h1);
    if (h2) pmReleaseCallbacks(h2);
    pmFinalize();
    std::sort(times.begin(), times.end());
    double mean = 0;
    for (double t : times) mean += t;
    mean /= times.size();
    std::printf("{\"flow\": \"%s\", \"n\": %llu, \"elems_per_subtask\": %llu, \"subtasks\": %lu, \"bits\": %d, "
                "\"steps\": %d, \"ms_per_flow\": %.3f, \"ms_min\": %.3f, \"check\": %s}\n",
                o.mode.c_str(), static_cast<unsigned long long>(o.n), static_cast<unsigned long long>(o.per), subtasks,
                o.bits, o.steps, mean, times.front(), ok ? "true" : "false");
    return ok ? 0 : 3;
}
