// Served mixed-size task stream over the pm:: API: the serving benchmark and
// its accuracy checks.
//
// Workload: N task submissions arriving as a Poisson stream of rate `rate`;
// a fraction `gemm_frac` are matrix products C = A*B (fp32 row-major, n
// log-uniform in [gemm_min, gemm_max]), the rest are unpivoted LU
// factorisations in place (fp32 column-major, n log-uniform in [lu_min,
// lu_max]) of uniform[-1,1] + n*I.  Sizes are rounded to multiples of 16.
// Every task reads its inputs from address spaces that stay resident on the
// device across tasks (a 8192x8192 A pool, a B pool and a 4096x4096 LU pool,
// uniform[-1,1] from fixed seeds; task i subscribes an n x n block at a random
// 16-byte-aligned offset) and writes its own output address space, which the
// client fetches to the host with pmFetchMemory; a task's latency runs from
// its arrival time to the moment its result is in host memory.  Each form uses
// the write-back policy that serves it best (measured): the served form leaves
// results on the device until the fetch thread's pmFetchMemory (copies overlap
// later tasks' kernels), the plain form has the runtime copy each result back
// on the task's own stream at task end (pmb_runtime_set_eager_writeback).
//
// Two forms run the same task list:
//  * served: tasks are submitted as they arrive and run concurrently -- the
//    runtime admits them by free slots and device memory, spreads them over
//    its compute streams and finishes each as soon as its own work is done; a
//    fetch thread copies results back while later tasks compute.  GEMM uses
//    the tcgen05 BF16x3 kernel, LU the FP64-panel / BF16x3-update kernel;
//    workspaces come from pmReserveCudaGlobalMem (the runtime's stream-ordered
//    pool), so nothing synchronises the device.
//  * plain: one task at a time (submit, wait, fetch, next), FP32 everywhere:
//    cuBLAS SGEMM -- the library call the reference's matrixMultiplyBlas GPU
//    callback makes (matrixMultiplyBlasCUDA.cu:54-77) -- or the FP32 SIMT
//    kernel of libpmb.so, and the blocked LU with FP32 SIMT GEMMs.
//
// After the timed stream, sampled tasks are checked: GEMM relative Frobenius
// error and LU ||A - LU||_F / ||A||_F against FP64, and (served form) each
// sampled result is recomputed with the task alone on the device and compared
// bit for bit with the result it produced inside the mix.
//
// Output: one JSON object on stdout.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pmPublicDefinitions.h"
#include "pmb_capi.h"

using namespace pm;

// Runtime counters exported by libpmlib.so.
extern "C" void pmb_runtime_stats(unsigned long long* h2d_bytes, unsigned long long* d2h_bytes,
                                  unsigned long long* gpu_subtasks, unsigned long long* batched_launches);
extern "C" void pmb_runtime_reset_stats(void);
extern "C" void pmb_runtime_set_eager_writeback(int on);
extern "C" double pmb_runtime_callback_seconds(void);
extern "C" void pmb_runtime_fetch_timers(double* host_s, double* wait_s, double* copy_s, unsigned long long* fetches);
extern "C" void pmb_runtime_admission(double* slot_wait_s, double* memory_wait_s, unsigned long long* evictions,
                                      unsigned long long* evicted_bytes);
extern "C" void pmb_runtime_timers(double* stub_s, double* admit_wait_s, double* pinned_alloc_s,
                                   unsigned long long* pinned_alloc_bytes);
extern "C" int sm_prepare_lu(const float* pool, int64_t ldp, float* out, int n, float diag, void* stream);
extern "C" double sm_gemm_rel_error(const float* dA, int64_t lda, const float* dB, int64_t ldb, const float* dC,
                                    int64_t ldc, int n);

namespace {

constexpr int kGemmPool = 8192;
constexpr int kLuPool = 4096;
constexpr int kLuNb = 64;

enum Kind { GEMM = 0, LU = 1 };
enum Mode { SERVED = 0, PLAIN = 1 };
enum PlainGemm { PLAIN_CUBLAS = 0, PLAIN_SIMT = 1 };

struct Spec {
    int kind, n;
    int ar, ac, br, bc;  // block origins in the pools (rows, columns)
    double t_arr;        // arrival, seconds after the stream starts
};

// taskConf of both task kinds (copied by the runtime at submission).
struct TaskConf {
    int kind, n, mode, plain_gemm;
    int ar, ac, br, bc;
    size_t ws_bytes;
};

struct Options {
    int tasks = 2000;
    double rate = 1000.0;
    uint64_t seed = 5;
    int gemm_min = 256, gemm_max = 8192, lu_min = 512, lu_max = 4096;
    double gemm_frac = 0.6;
    int warmup = 256;
    int check = 16;
    bool run_served = true, run_plain = true;
    int plain_gemm = PLAIN_CUBLAS;
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
double unit(uint64_t& s) { return (splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

// uniform[-1,1) fill, parallel over host threads, deterministic per element.
void fill_uniform(float* p, size_t count, uint64_t seed) {
    const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([=] {
            for (size_t i = t; i < count; i += nt) {
                uint64_t s = seed * 0x100000001B3ull + i;
                p[i] = static_cast<float>(unit(s) * 2.0 - 1.0);
            }
        });
    for (auto& x : th) x.join();
}

int round16(double x) { return std::max(16, static_cast<int>(std::lround(x / 16.0)) * 16); }

std::vector<Spec> make_specs(const Options& o, int count, uint64_t seed, double rate) {
    std::vector<Spec> v(count);
    uint64_t s = seed;
    double t = 0;
    for (int i = 0; i < count; ++i) {
        Spec& x = v[i];
        x.kind = unit(s) < o.gemm_frac ? GEMM : LU;
        const int lo = x.kind == GEMM ? o.gemm_min : o.lu_min, hi = x.kind == GEMM ? o.gemm_max : o.lu_max;
        x.n = std::min(hi, round16(std::exp(std::log(lo) + unit(s) * (std::log(hi) - std::log(lo)))));
        const int pool = x.kind == GEMM ? kGemmPool : kLuPool;
        const int span = pool - x.n;
        x.ar = static_cast<int>(unit(s) * (span + 1));
        x.ac = static_cast<int>(unit(s) * (span / 4 + 1)) * 4;  // 16-byte aligned block start
        x.br = static_cast<int>(unit(s) * (span + 1));
        x.bc = static_cast<int>(unit(s) * (span / 4 + 1)) * 4;
        if (x.kind == LU) x.ar = x.ar / 4 * 4;                   // column-major: rows are contiguous
        t += rate > 0 ? -std::log(1.0 - unit(s)) / rate : 0.0;
        x.t_arr = t;
    }
    return v;
}

// ---------------------------------------------------------------------------
// pm:: callbacks

cublasHandle_t g_cublas = nullptr;
std::mutex g_cublas_mu;

pmStatus mix_dd(pmTaskInfo ti, pmDeviceInfo dev, pmSubtaskInfo si) {
    const TaskConf* c = static_cast<const TaskConf*>(ti.taskConf);
    const size_t n = static_cast<size_t>(c->n);
    pmStatus st;
    if (c->kind == GEMM) {
        const size_t ld = kGemmPool;
        st = pmSubscribeToMemory(ti.taskHandle, dev.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION,
                                 pmScatteredSubscriptionInfo((c->ar * ld + c->ac) * 4, n * 4, ld * 4, n));
        if (st == pmSuccess)
            st = pmSubscribeToMemory(ti.taskHandle, dev.deviceHandle, si.subtaskId, si.splitInfo, 1, READ_SUBSCRIPTION,
                                     pmScatteredSubscriptionInfo((c->br * ld + c->bc) * 4, n * 4, ld * 4, n));
        if (st == pmSuccess)
            st = pmSubscribeToMemory(ti.taskHandle, dev.deviceHandle, si.subtaskId, si.splitInfo, 2,
                                     WRITE_SUBSCRIPTION, pmSubscriptionInfo(0, n * n * 4));
    } else {
        const size_t ld = kLuPool;  // column-major pool: column c of the block starts at (ac + c) * ld + ar
        st = pmSubscribeToMemory(ti.taskHandle, dev.deviceHandle, si.subtaskId, si.splitInfo, 0, READ_SUBSCRIPTION,
                                 pmScatteredSubscriptionInfo((c->ac * ld + c->ar) * 4, n * 4, ld * 4, n));
        if (st == pmSuccess)
            st = pmSubscribeToMemory(ti.taskHandle, dev.deviceHandle, si.subtaskId, si.splitInfo, 1,
                                     WRITE_SUBSCRIPTION, pmSubscriptionInfo(0, n * n * 4));
    }
    if (st == pmSuccess && c->ws_bytes)
        st = pmReserveCudaGlobalMem(ti.taskHandle, dev.deviceHandle, si.subtaskId, si.splitInfo, c->ws_bytes);
    return st;
}

pmStatus mix_gpu(pmTaskInfo ti, pmDeviceInfo, pmSubtaskInfo si, void* stream) {
    const TaskConf* c = static_cast<const TaskConf*>(ti.taskConf);
    const int n = c->n;
    void* ws = si.gpuContext.reservedGlobalMem;
    int st = PMB_SUCCESS;
    if (c->kind == GEMM) {
        const float* A = static_cast<const float*>(si.memInfo[0].ptr);
        const float* B = static_cast<const float*>(si.memInfo[1].ptr);
        float* C = static_cast<float*>(si.memInfo[2].ptr);
        if (c->mode == SERVED) {
            st = pmb_sgemm_bf16x3(n, n, n, 1.0f, A, kGemmPool, B, kGemmPool, 0.0f, C, n, ws, c->ws_bytes, stream);
        } else if (c->plain_gemm == PLAIN_SIMT) {
            st = pmb_sgemm_plain(n, n, n, 1.0f, A, kGemmPool, B, kGemmPool, 0.0f, C, n, stream);
        } else {
            // Row-major C = A*B is column-major C^T = B^T * A^T.
            std::lock_guard<std::mutex> g(g_cublas_mu);
            const float one = 1.0f, zero = 0.0f;
            if (cublasSetStream(g_cublas, static_cast<cudaStream_t>(stream)) != CUBLAS_STATUS_SUCCESS ||
                cublasSgemm(g_cublas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, B, kGemmPool, A, kGemmPool, &zero, C,
                            n) != CUBLAS_STATUS_SUCCESS)
                return pmGraphicsCardError;
        }
    } else {
        const float* P = static_cast<const float*>(si.memInfo[0].ptr);
        float* M = static_cast<float*>(si.memInfo[1].ptr);
        if (sm_prepare_lu(P, kLuPool, M, n, static_cast<float>(n), stream) != 0) return pmGraphicsCardError;
        st = c->mode == SERVED ? pmb_lu_decompose(M, n, n, kLuNb, ws, c->ws_bytes, stream)
                               : pmb_lu_decompose_plain(M, n, n, kLuNb, ws, c->ws_bytes, stream);
    }
    return st == PMB_SUCCESS ? pmSuccess : static_cast<pmStatus>(st);
}

// ---------------------------------------------------------------------------
// running a task list

struct Pools {
    pmMemHandle a = nullptr, b = nullptr, lu = nullptr;
    float *ha = nullptr, *hb = nullptr, *hlu = nullptr;
};

struct Run {
    std::vector<double> done;      // completion (result on the host), seconds after start
    double fetch_busy = 0;         // seconds the client spent in pmFetchMemory
    std::vector<int> sampled;      // task indices whose outputs are kept
    std::map<int, std::vector<float>> outputs;
    double wall = 0;
    std::string error;
};

struct Client {
    pmCallbackHandle cb = nullptr;
    Pools pools;
    Options opt;
};

Client g_client;

// Completed tasks handed from the completion callback to the fetch thread.
std::mutex g_done_mu;
std::condition_variable g_done_cv;
std::deque<uint64_t> g_done;

pmStatus on_complete(pmTaskInfo ti) {
    {
        std::lock_guard<std::mutex> g(g_done_mu);
        g_done.push_back(ti.taskId);
    }
    g_done_cv.notify_one();
    return pmSuccess;
}

TaskConf conf_of(const Spec& s, int mode, int plain_gemm) {
    TaskConf c;
    c.kind = s.kind;
    c.n = s.n;
    c.mode = mode;
    c.plain_gemm = plain_gemm;
    c.ar = s.ar;
    c.ac = s.ac;
    c.br = s.br;
    c.bc = s.bc;
    if (s.kind == GEMM)
        c.ws_bytes = mode == SERVED ? pmb_gemm_workspace_bytes(s.n, s.n, s.n) : 0;
    else
        c.ws_bytes = pmb_lu_workspace_bytes(s.n, kLuNb);
    return c;
}

struct Live {
    std::atomic<pmTaskHandle> task{nullptr};  // stored by the submitter, read by the fetch thread
    pmMemHandle out = nullptr;
    TaskConf conf;
    pmTaskMem mem[3];
};

// Creates the task's output address space and submits it; the handle is
// published last (release), after `out` and `conf`.
bool submit(const Spec& s, int mode, uint64_t id, Live& L) {
    const Pools& p = g_client.pools;
    L.conf = conf_of(s, mode, g_client.opt.plain_gemm);
    const size_t bytes = static_cast<size_t>(s.n) * s.n * 4;
    if (pmCreateMemory(bytes, &L.out) != pmSuccess) return false;
    uint count;
    if (s.kind == GEMM) {
        L.mem[0] = pmTaskMem(p.a, READ_ONLY, SUBSCRIPTION_NATURAL);
        L.mem[1] = pmTaskMem(p.b, READ_ONLY, SUBSCRIPTION_NATURAL);
        L.mem[2] = pmTaskMem(L.out, WRITE_ONLY, SUBSCRIPTION_NATURAL);
        count = 3;
    } else {
        L.mem[0] = pmTaskMem(p.lu, READ_ONLY, SUBSCRIPTION_NATURAL);
        L.mem[1] = pmTaskMem(L.out, WRITE_ONLY, SUBSCRIPTION_NATURAL);
        count = 2;
    }
    pmTaskDetails d(&L.conf, sizeof(TaskConf), L.mem, count, g_client.cb, 1);
    d.taskId = id;
    d.policy = NODE_EQUAL_STATIC;
    pmTaskHandle h = nullptr;
    if (pmSubmitTask(d, &h) != pmSuccess) return false;
    L.task.store(h, std::memory_order_release);
    return true;
}

// Fetch a finished task's result to the host, keep it if sampled, release.
bool collect(Live& L, int idx, bool keep, Run& r, double t0) {
    const double f0 = now_s();
    if (pmFetchMemory(L.out) != pmSuccess) return false;
    r.fetch_busy += now_s() - f0;
    if (keep) {
        void* hp = nullptr;
        pmGetRawMemPtr(L.out, &hp);
        const size_t elems = static_cast<size_t>(L.conf.n) * L.conf.n;
        r.outputs[idx].assign(static_cast<float*>(hp), static_cast<float*>(hp) + elems);
    }
    r.done[idx] = now_s() - t0;
    const pmStatus ts = pmReleaseTask(L.task.load());
    pmReleaseMemory(L.out);
    L.task = nullptr;
    L.out = nullptr;
    return ts == pmSuccess;
}

void sleep_until(double t) {
    const double d = t - now_s();
    if (d > 0) std::this_thread::sleep_for(std::chrono::duration<double>(d));
}

Run run_stream(const std::vector<Spec>& specs, int mode, const std::vector<int>& sampled, bool honour_arrivals) {
    Run r;
    const int N = static_cast<int>(specs.size());
    r.done.assign(N, -1.0);
    r.sampled = sampled;
    std::vector<char> keep(N, 0);
    for (int i : sampled) keep[i] = 1;
    std::vector<Live> live(N);
    {
        std::lock_guard<std::mutex> g(g_done_mu);
        g_done.clear();
    }
    const double t0 = now_s();
    if (mode == PLAIN) {
        for (int i = 0; i < N; ++i) {
            if (honour_arrivals) sleep_until(t0 + specs[i].t_arr);
            if (!submit(specs[i], mode, i, live[i]) || pmWaitForTaskCompletion(live[i].task.load()) != pmSuccess ||
                !collect(live[i], i, keep[i], r, t0)) {
                r.error = std::string("task ") + std::to_string(i) + ": " + pmGetLastError();
                return r;
            }
        }
        {
            std::lock_guard<std::mutex> g(g_done_mu);
            g_done.clear();
        }
    } else {
        std::atomic<bool> failed{false};
        std::string fetch_err;
        std::thread fetcher([&] {
            for (int got = 0; got < N && !failed;) {
                uint64_t id;
                {
                    std::unique_lock<std::mutex> lk(g_done_mu);
                    if (!g_done_cv.wait_for(lk, std::chrono::seconds(120), [] { return !g_done.empty(); })) {
                        fetch_err = "no task completed for 120 s";
                        failed = true;
                        return;
                    }
                    id = g_done.front();
                    g_done.pop_front();
                }
                const int i = static_cast<int>(id);
                while (!live[i].task.load(std::memory_order_acquire)) std::this_thread::yield();
                if (!collect(live[i], i, keep[i], r, t0)) {
                    fetch_err = std::string("task ") + std::to_string(i) + ": " + pmGetLastError();
                    failed = true;
                    return;
                }
                ++got;
            }
        });
        for (int i = 0; i < N && !failed; ++i) {
            if (honour_arrivals) sleep_until(t0 + specs[i].t_arr);
            if (!submit(specs[i], mode, i, live[i])) {
                r.error = std::string("submit ") + std::to_string(i) + ": " + pmGetLastError();
                failed = true;
                break;
            }
        }
        fetcher.join();
        if (r.error.empty()) r.error = fetch_err;
    }
    r.wall = now_s() - t0;
    return r;
}

// ---------------------------------------------------------------------------
// accuracy checks (device copies of the pools, FP64 kernels)

struct DevPools {
    float *a = nullptr, *b = nullptr, *lu = nullptr;
};

double gemm_error(const DevPools& dp, const Spec& s, const std::vector<float>& C) {
    float* dC = nullptr;
    const size_t bytes = static_cast<size_t>(s.n) * s.n * 4;
    if (cudaMalloc(&dC, bytes) != cudaSuccess) return -1;
    cudaMemcpy(dC, C.data(), bytes, cudaMemcpyHostToDevice);
    const double e = sm_gemm_rel_error(dp.a + static_cast<size_t>(s.ar) * kGemmPool + s.ac, kGemmPool,
                                       dp.b + static_cast<size_t>(s.br) * kGemmPool + s.bc, kGemmPool, dC, s.n, s.n);
    cudaFree(dC);
    return e;
}

double lu_residual(const DevPools& dp, const Spec& s, const std::vector<float>& LUh) {
    float *dA = nullptr, *dLU = nullptr;
    double* sums = nullptr;
    const size_t bytes = static_cast<size_t>(s.n) * s.n * 4;
    if (cudaMalloc(&dA, bytes) != cudaSuccess || cudaMalloc(&dLU, bytes) != cudaSuccess ||
        cudaMalloc(&sums, 16) != cudaSuccess)
        return -1;
    sm_prepare_lu(dp.lu + static_cast<size_t>(s.ac) * kLuPool + s.ar, kLuPool, dA, s.n, static_cast<float>(s.n),
                  nullptr);
    cudaMemcpy(dLU, LUh.data(), bytes, cudaMemcpyHostToDevice);
    double h[2] = {0, 0};
    if (pmb_lu_residual_f64(dA, s.n, dLU, s.n, s.n, sums, nullptr) == PMB_SUCCESS)
        cudaMemcpy(h, sums, 16, cudaMemcpyDeviceToHost);
    cudaFree(dA);
    cudaFree(dLU);
    cudaFree(sums);
    return h[1] > 0 ? std::sqrt(h[0] / h[1]) : -1;
}

std::string esc(const std::string& in) {
    std::string o;
    for (char ch : in) {
        if (ch == '"' || ch == '\\') o += '\\';
        o += (ch == '\n' || ch == '\t') ? ' ' : ch;
    }
    return o;
}

double pct(std::vector<double> v, double p) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    const double k = p / 100.0 * (v.size() - 1);
    const size_t lo = static_cast<size_t>(std::floor(k)), hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (v[hi] - v[lo]) * (k - lo);
}

std::string stream_json(const char* name, const std::vector<Spec>& specs, const Run& r, const DevPools& dp,
                        double* tasks_per_s, double* max_gemm_err, double* max_lu_res) {
    std::vector<double> lat, lat_g, lat_l;
    double last = 0;
    for (size_t i = 0; i < specs.size(); ++i) {
        if (r.done[i] < 0) continue;
        const double l = r.done[i] - specs[i].t_arr;
        lat.push_back(l);
        (specs[i].kind == GEMM ? lat_g : lat_l).push_back(l);
        last = std::max(last, r.done[i]);
    }
    *tasks_per_s = last > 0 ? lat.size() / last : 0;
    *max_gemm_err = 0;
    *max_lu_res = 0;
    std::string checks;
    for (int i : r.sampled) {
        auto it = r.outputs.find(i);
        if (it == r.outputs.end()) continue;
        const Spec& s = specs[i];
        const double e = s.kind == GEMM ? gemm_error(dp, s, it->second) : lu_residual(dp, s, it->second);
        if (s.kind == GEMM) *max_gemm_err = std::max(*max_gemm_err, e);
        else *max_lu_res = std::max(*max_lu_res, e);
        char b[160];
        snprintf(b, sizeof(b), "%s{\"task\": %d, \"kind\": \"%s\", \"n\": %d, \"%s\": %.3e}", checks.empty() ? "" : ", ",
                 i, s.kind == GEMM ? "gemm" : "lu", s.n, s.kind == GEMM ? "rel_err" : "residual", e);
        checks += b;
    }
    char buf[1024];
    snprintf(buf, sizeof(buf),
             "\"%s\": {\"tasks_per_s\": %.2f, \"completed\": %zu, \"span_s\": %.4f, \"p50_ms\": %.3f, \"p99_ms\": %.3f, "
             "\"gemm_p50_ms\": %.3f, \"gemm_p99_ms\": %.3f, \"lu_p50_ms\": %.3f, \"lu_p99_ms\": %.3f, "
             "\"max_gemm_rel_err\": %.3e, \"max_lu_residual\": %.3e, \"fetch_busy_s\": %.4f, \"error\": \"%s\", "
             "\"checks\": [",
             name, *tasks_per_s, lat.size(), last, 1e3 * pct(lat, 50), 1e3 * pct(lat, 99), 1e3 * pct(lat_g, 50),
             1e3 * pct(lat_g, 99), 1e3 * pct(lat_l, 50), 1e3 * pct(lat_l, 99), *max_gemm_err, *max_lu_res,
             r.fetch_busy, esc(r.error).c_str());
    return std::string(buf) + checks + "]}";
}

int usage() {
    fprintf(stderr,
            "usage: served_mix [--tasks N] [--rate R] [--seed S] [--gemm-min n] [--gemm-max n] [--lu-min n] "
            "[--lu-max n] [--gemm-frac f] [--warmup W] [--check K] [--mode served|plain|both] "
            "[--plain-gemm cublas|simt]\n");
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    Options& o = g_client.opt;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() -> const char* { return i + 1 < argc ? argv[++i] : ""; };
        if (a == "--tasks") o.tasks = atoi(val());
        else if (a == "--rate") o.rate = atof(val());
        else if (a == "--seed") o.seed = strtoull(val(), nullptr, 10);
        else if (a == "--gemm-min") o.gemm_min = atoi(val());
        else if (a == "--gemm-max") o.gemm_max = atoi(val());
        else if (a == "--lu-min") o.lu_min = atoi(val());
        else if (a == "--lu-max") o.lu_max = atoi(val());
        else if (a == "--gemm-frac") o.gemm_frac = atof(val());
        else if (a == "--warmup") o.warmup = atoi(val());
        else if (a == "--check") o.check = atoi(val());
        else if (a == "--mode") {
            const std::string m = val();
            o.run_served = m != "plain";
            o.run_plain = m != "served";
        } else if (a == "--plain-gemm") o.plain_gemm = std::string(val()) == "simt" ? PLAIN_SIMT : PLAIN_CUBLAS;
        else return usage();
    }
    if (o.tasks < 1 || o.gemm_min < 16 || o.gemm_max > kGemmPool || o.gemm_min > o.gemm_max || o.lu_min < 16 ||
        o.lu_max > kLuPool || o.lu_min > o.lu_max)
        return usage();

    if (pmInitialize() != pmSuccess) {
        printf("{\"error\": \"pmInitialize: %s\"}\n", esc(pmGetLastError()).c_str());
        return 1;
    }
    if (cublasCreate(&g_cublas) != CUBLAS_STATUS_SUCCESS) {
        printf("{\"error\": \"cublasCreate failed\"}\n");
        return 1;
    }
    pmCallbacks cb;
    cb.dataDistribution = mix_dd;
    cb.subtask_gpu_custom = mix_gpu;
    cb.taskCompletionCallback = on_complete;
    if (pmRegisterCallbacks("servedMix", cb, &g_client.cb) != pmSuccess) return 1;

    // Resident input pools.
    Pools& p = g_client.pools;
    const size_t gbytes = static_cast<size_t>(kGemmPool) * kGemmPool * 4, lbytes = static_cast<size_t>(kLuPool) * kLuPool * 4;
    pmCreateMemory(gbytes, &p.a);
    pmCreateMemory(gbytes, &p.b);
    pmCreateMemory(lbytes, &p.lu);
    void* hp;
    pmGetRawMemPtr(p.a, &hp);
    p.ha = static_cast<float*>(hp);
    pmGetRawMemPtr(p.b, &hp);
    p.hb = static_cast<float*>(hp);
    pmGetRawMemPtr(p.lu, &hp);
    p.hlu = static_cast<float*>(hp);
    fill_uniform(p.ha, gbytes / 4, 11);
    fill_uniform(p.hb, gbytes / 4, 12);
    fill_uniform(p.hlu, lbytes / 4, 13);
    DevPools dp;
    cudaMalloc(&dp.a, gbytes);
    cudaMalloc(&dp.b, gbytes);
    cudaMalloc(&dp.lu, lbytes);
    cudaMemcpy(dp.a, p.ha, gbytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dp.b, p.hb, gbytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dp.lu, p.hlu, lbytes, cudaMemcpyHostToDevice);

    const std::vector<Spec> specs = make_specs(o, o.tasks, o.seed, o.rate);
    // Warm-up list: the two largest tasks (they make the whole pools resident)
    // plus tasks of the same distribution, all submitted at once.
    std::vector<Spec> warm = make_specs(o, std::max(o.warmup, 2), o.seed + 1000, 0.0);
    warm[0].kind = GEMM;
    warm[0].n = o.gemm_max;
    warm[0].ar = warm[0].ac = warm[0].br = warm[0].bc = 0;
    warm[1].kind = LU;
    warm[1].n = o.lu_max;
    warm[1].ar = warm[1].ac = 0;
    // Sampled tasks for the checks: evenly spread over the list.
    std::vector<int> sampled;
    for (int k = 0; k < o.check && k < o.tasks; ++k) sampled.push_back(static_cast<int>((static_cast<long long>(k) * o.tasks) / o.check));

    double gemm_flop = 0, lu_flop = 0, out_bytes = 0;
    int n_gemm = 0;
    for (const Spec& s : specs) {
        const double n = s.n;
        if (s.kind == GEMM) {
            gemm_flop += 2 * n * n * n;
            ++n_gemm;
        } else {
            lu_flop += 2.0 / 3.0 * n * n * n;
        }
        out_bytes += 4 * n * n;
    }

    std::string js = "{";
    char head[768];
    snprintf(head, sizeof(head),
             "\"workload\": \"served mixed-size stream: %d tasks, Poisson arrivals %.1f/s, %.0f%% GEMM n in [%d,%d], "
             "%.0f%% LU n in [%d,%d], log-uniform, multiples of 16\", \"tasks\": %d, \"gemm_tasks\": %d, \"lu_tasks\": %d, "
             "\"rate_per_s\": %.2f, \"gemm_gflop\": %.1f, \"lu_gflop\": %.1f, \"result_bytes\": %.0f, \"plain_gemm\": \"%s\"",
             o.tasks, o.rate, 100 * o.gemm_frac, o.gemm_min, o.gemm_max, 100 * (1 - o.gemm_frac), o.lu_min, o.lu_max,
             o.tasks, n_gemm, o.tasks - n_gemm, o.rate, gemm_flop / 1e9, lu_flop / 1e9, out_bytes,
             o.plain_gemm == PLAIN_SIMT ? "libpmb FP32 SIMT" : "cuBLAS SGEMM FP32");
    js += head;

    double served_tps = 0, plain_tps = 0, ge, lr;
    if (o.run_served) {
        pmb_runtime_set_eager_writeback(0);
        const Run w = run_stream(warm, SERVED, {}, false);
        if (!w.error.empty()) {
            printf("{\"error\": \"served warm-up: %s\"}\n", esc(w.error).c_str());
            return 1;
        }
        pmb_runtime_reset_stats();
        const Run r = run_stream(specs, SERVED, sampled, true);
        unsigned long long h2d = 0, d2h = 0, subs = 0, bat = 0, pin_b = 0;
        double stub_s = 0, admit_s = 0, pin_s = 0, slot_s = 0, mem_s = 0;
        unsigned long long ev = 0, ev_b = 0;
        pmb_runtime_stats(&h2d, &d2h, &subs, &bat);
        pmb_runtime_timers(&stub_s, &admit_s, &pin_s, &pin_b);
        pmb_runtime_admission(&slot_s, &mem_s, &ev, &ev_b);
        const double cb_s = pmb_runtime_callback_seconds();
        double fh_s = 0, fw_s = 0, fc_s = 0;
        unsigned long long nfetch = 0;
        pmb_runtime_fetch_timers(&fh_s, &fw_s, &fc_s, &nfetch);
        js += ", " + stream_json("served", specs, r, dp, &served_tps, &ge, &lr);
        // Alone vs. in the mix: recompute each sampled task by itself.
        int same = 0, compared = 0;
        for (int i : sampled) {
            auto it = r.outputs.find(i);
            if (it == r.outputs.end()) continue;
            const Run a = run_stream({specs[i]}, SERVED, {0}, false);
            auto jt = a.outputs.find(0);
            if (jt == a.outputs.end()) continue;
            ++compared;
            if (jt->second.size() == it->second.size() &&
                std::memcmp(jt->second.data(), it->second.data(), 4 * it->second.size()) == 0)
                ++same;
        }
        char b[1024];
        snprintf(b, sizeof(b), ", \"served_alone_vs_mix\": {\"compared\": %d, \"bit_identical\": %d}, "
                               "\"served_h2d_bytes\": %llu, \"served_d2h_bytes\": %llu, \"served_runtime\": "
                               "{\"stub_issue_s\": %.4f, \"admission_wait_s\": %.4f, \"slot_wait_s\": %.4f, "
                               "\"memory_wait_s\": %.4f, \"evictions\": %llu, \"evicted_bytes\": %llu, "
                               "\"pinned_alloc_s\": %.4f, \"pinned_alloc_bytes\": %llu, \"callback_s\": %.4f, "
                               "\"fetches\": %llu, \"fetch_host_s\": %.4f, \"fetch_wait_s\": %.4f, \"fetch_copy_s\": %.4f}",
                 compared, same, h2d, d2h, stub_s, admit_s, slot_s, mem_s, ev, ev_b, pin_s, pin_b, cb_s, nfetch, fh_s,
                 fw_s, fc_s);
        js += b;
    }
    if (o.run_plain) {
        pmb_runtime_set_eager_writeback(1);
        const Run w = run_stream(warm, PLAIN, {}, false);
        if (!w.error.empty()) {
            printf("{\"error\": \"plain warm-up: %s\"}\n", esc(w.error).c_str());
            return 1;
        }
        const Run r = run_stream(specs, PLAIN, sampled, true);
        js += ", " + stream_json("plain", specs, r, dp, &plain_tps, &ge, &lr);
    }
    if (o.run_served && o.run_plain && plain_tps > 0) {
        char b[96];
        snprintf(b, sizeof(b), ", \"served_over_plain\": %.3f", served_tps / plain_tps);
        js += b;
    }
    js += "}";
    printf("%s\n", js.c_str());
    fflush(stdout);
    cudaFree(dp.a);
    cudaFree(dp.b);
    cudaFree(dp.lu);
    cublasDestroy(g_cublas);
    pmReleaseMemory(p.a);
    pmReleaseMemory(p.b);
    pmReleaseMemory(p.lu);
    pmFinalize();
    return 0;
}
