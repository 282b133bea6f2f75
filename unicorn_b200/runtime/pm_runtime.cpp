// pm:: runtime of the B200 subtask path (libpmlib.so).
//
// Implements the public API of pmPublicDefinitions.h / pmPublicUtilities.h for
// one process and one CUDA device.  The reference spreads this over pmController,
// pmTask*, pmScheduler, pmSubscriptionManager, pmExecutionStub and
// pmCudaInterface (source/code/src/); here it is one in-process controller
// with two worker threads:
//
//  * the CUDA execution stub (replaces pmStubCUDA::Execute and its helpers,
//    pmExecutionStub.cpp:2980-4042): runs each task's data-distribution
//    callback for every subtask, turns the recorded subscriptions into device
//    views, stages the missing bytes into a device-resident mirror of every
//    address space (one 2-D copy per scattered subscription, on a dedicated
//    copy stream), launches each subtask's GPU callback on the next of
//    PMB_STREAMS (default 16) compute streams, round robin across tasks, and
//    keeps results on the device.  Tasks are issued back to back: dependencies
//    between tasks that share address spaces are CUDA events, never host
//    waits, so independent tasks overlap on the device.  A task is admitted
//    when one of PMB_MAX_INFLIGHT (default 64) slots is free and its device
//    memory fits; otherwise the stub waits for in-flight tasks to finish;
//  * the completion thread: polls the in-flight tasks' completion events,
//    finishes each task as soon as its own work is done (out of issue order),
//    runs the completion callback and wakes waiters.
//
// Address spaces keep a pinned host copy and, once a GPU task has used them,
// a full device mirror.  Coherence is tracked per byte range: dev_valid (the
// device copy is current) and host_stale (the device is newer than the host,
// written back by pmFetchMemory).  This is the analogue of the reference's
// CUDA cache (pmCache, pmExecutionStub.cpp:3022-3070) at address-space
// granularity; with the cache disabled (pmTaskDetails::cudaCacheEnabled or
// PMLIB_DISABLE_CUDA_CACHE) writes go back to the host at task end and the
// device copy is dropped.
//
// All CUDA work goes through the C ABI of libpmb.so (pmb_capi.h).
#include "pm_runtime.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <set>

#include "pmb_capi.h"

namespace pmr {

// ---------------------------------------------------------------------------
// errors

static thread_local std::string t_last_error;

static pmStatus fail(pmStatus st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return st;
}

// Map a non-zero libpmb status to pmStatus (same numbering) and keep its message.
static pmStatus dev_fail(int st, const char* what) {
    return fail(static_cast<pmStatus>(st), "%s: %s", what, pmb_last_error());
}

#define PMR_DEV(call)                                            \
    do {                                                         \
        const int pmr_st_ = (call);                              \
        if (pmr_st_ != PMB_SUCCESS) return dev_fail(pmr_st_, #call); \
    } while (0)

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static unsigned long long ns_since(double t0) { return static_cast<unsigned long long>((now_s() - t0) * 1e9); }

static bool env_flag(const char* name) {
    const char* v = getenv(name);
    return v && atoi(v) != 0;
}

// ---------------------------------------------------------------------------
// RangeSet

void RangeSet::add(size_t lo, size_t hi) {
    if (lo >= hi) return;
    auto it = m_.upper_bound(lo);
    if (it != m_.begin()) {
        auto prev = std::prev(it);
        if (prev->second >= lo) {
            lo = prev->first;
            hi = std::max(hi, prev->second);
            it = m_.erase(prev);
        }
    }
    while (it != m_.end() && it->first <= hi) {
        hi = std::max(hi, it->second);
        it = m_.erase(it);
    }
    m_[lo] = hi;
}

void RangeSet::remove(size_t lo, size_t hi) {
    if (lo >= hi) return;
    auto it = m_.upper_bound(lo);
    if (it != m_.begin()) --it;
    std::vector<std::pair<size_t, size_t>> keep;
    while (it != m_.end() && it->first < hi) {
        if (it->second <= lo) {
            ++it;
            continue;
        }
        if (it->first < lo) keep.emplace_back(it->first, lo);
        if (it->second > hi) keep.emplace_back(hi, it->second);
        it = m_.erase(it);
    }
    for (auto& k : keep) m_[k.first] = k.second;
}

bool RangeSet::covers(size_t lo, size_t hi) const {
    if (lo >= hi) return true;
    auto it = m_.upper_bound(lo);
    if (it == m_.begin()) return false;
    --it;
    return it->first <= lo && it->second >= hi;
}

void RangeSet::missing(size_t lo, size_t hi, std::vector<std::pair<size_t, size_t>>& out) const {
    size_t cur = lo;
    auto it = m_.upper_bound(lo);
    if (it != m_.begin()) --it;
    for (; it != m_.end() && it->first < hi; ++it) {
        if (it->second <= cur) continue;
        if (it->first > cur) out.emplace_back(cur, std::min(it->first, hi));
        cur = std::max(cur, it->second);
        if (cur >= hi) break;
    }
    if (cur < hi) out.emplace_back(cur, hi);
}

void RangeSet::present(size_t lo, size_t hi, std::vector<std::pair<size_t, size_t>>& out) const {
    auto it = m_.upper_bound(lo);
    if (it != m_.begin()) --it;
    for (; it != m_.end() && it->first < hi; ++it) {
        const size_t a = std::max(lo, it->first), b = std::min(hi, it->second);
        if (a < b) out.emplace_back(a, b);
    }
}

size_t RangeSet::bytes() const {
    size_t b = 0;
    for (auto& kv : m_) b += kv.second - kv.first;
    return b;
}

// ---------------------------------------------------------------------------
// controller state

struct Stats {
    std::atomic<unsigned long long> h2d{0}, d2h{0}, gpu_subtasks{0}, batched{0};
    // nanoseconds: stub thread issuing tasks, stub waiting for admission, pinned allocation
    std::atomic<unsigned long long> stub_ns{0}, admit_ns{0}, pin_ns{0}, pin_bytes{0};
    // admission: waiting for a slot, waiting for memory; mirrors evicted to make room
    std::atomic<unsigned long long> slot_ns{0}, mem_ns{0}, evictions{0}, evicted_bytes{0};
    std::atomic<unsigned long long> callback_ns{0};  // inside GPU callbacks (the apps' launches)
    // subtask copies sent to the host sentinel-compressed, and the bytes they took
    std::atomic<unsigned long long> sentinel_copies{0}, sentinel_bytes{0};
    // write-back (pmFetchMemory and friends): host buffer, waiting for the
    // producing task's event, the copies themselves
    std::atomic<unsigned long long> fetch_host_ns{0}, fetch_wait_ns{0}, fetch_copy_ns{0}, fetches{0};
};

static unsigned long long ns_since(double t0);

struct Controller {
    std::mutex mu;  // registries
    bool initialized = false;
    bool has_gpu = false;
    int device = 0;
    pmDeviceInfo gpu_info, cpu_info;
    void* dev_device_info = nullptr;
    void* dev_status = nullptr;
    std::vector<std::unique_ptr<CallbackSet>> callbacks;
    std::set<AddressSpace*> spaces;
    std::set<Task*> tasks;
    struct BatchHook {
        BatchFn fn = nullptr;
        size_t groups = 0;  // launches per task; 0: batch_groups
    };
    std::map<void*, BatchHook> batch;
    // stub
    std::thread stub, completer;
    std::mutex qmu;
    std::condition_variable qcv;
    std::deque<Task*> queue;
    std::deque<Task*> inflight;
    std::condition_variable icv;
    bool stopping = false;
    void* copy_stream = nullptr;
    std::vector<void*> streams;
    std::atomic<uint64_t> next_stream{0};  // compute streams are handed out round robin
    void* fetch_stream = nullptr;
    size_t reserve_bytes = 0;
    // Device memory the runtime may hold (mirrors + reserved subtask memory):
    // free memory at initialisation minus the reserve, with 10 % headroom for
    // pool fragmentation.  Admission is decided against this budget and the
    // runtime's own count, not by querying the device per task.
    int64_t dev_budget = 0;
    std::atomic<int64_t> dev_held{0};
    size_t max_inflight = 64;              // GPU tasks on the device at once (admission slots)
    std::atomic<bool> eager_writeback{false};  // copy written bytes to the host at task end
    size_t batch_groups = 16;              // launches a batched task is split into (pipelined staging)
    bool batch_off = false;                // PMB_NO_BATCH: every subtask through its own callback
    // pinned host buffers of released address spaces, kept for reuse
    std::mutex pin_mu;
    std::multimap<size_t, char*> pin_free;
    size_t pin_cached = 0, pin_limit = 0;
    std::atomic<uint64_t> lru{0};
    Stats stats;
    // memory-mapped files
    std::map<std::string, std::pair<void*, size_t>> files;
};

// Never destroyed: an app that exits without pmFinalize (exit() on an error
// path) must not run the destructors of condition variables the stub and
// completer threads still wait on, which would block the exit.
static Controller& ctl() {
    static Controller* c = new Controller;
    return *c;
}

void register_batch(pmSubtaskCallback_GPU_Custom callback, BatchFn batch, size_t groups) {
    std::lock_guard<std::mutex> g(ctl().mu);
    ctl().batch[reinterpret_cast<void*>(callback)] = Controller::BatchHook{batch, groups};
}

// Data-distribution context of the calling thread.
struct DdContext {
    Task* task = nullptr;
};
static thread_local DdContext t_dd;

static Task* task_of(pmTaskHandle h) {
    Controller& c = ctl();
    std::lock_guard<std::mutex> g(c.mu);
    Task* t = static_cast<Task*>(h);
    return c.tasks.count(t) ? t : nullptr;
}

static AddressSpace* space_of(pmMemHandle h) {
    Controller& c = ctl();
    std::lock_guard<std::mutex> g(c.mu);
    AddressSpace* a = static_cast<AddressSpace*>(h);
    return c.spaces.count(a) && !a->released ? a : nullptr;
}

// Host copies are allocated on first host use (pmGetRawMemPtr, a fetch, a CPU
// task, a write-back): an address space only the GPU ever touches never costs
// a pinned allocation.  Called with a->mu held (or before the space is shared).
//
// Pinned allocations are expensive (page locking, and freeing one synchronises
// the device), so they come in size classes -- 64 KiB, then four classes per
// power of two, at most 25 % above the request -- and buffers of released
// address spaces are cached per class, up to PMB_PINNED_CACHE_BYTES (default
// 16 GiB), for the next address space of the same class.
static size_t pin_class(size_t len) {
    if (len <= (size_t(64) << 10)) return size_t(64) << 10;
    size_t p = 1;
    while (p < len) p <<= 1;
    size_t cls = p / 2;
    while (cls < len) cls += p / 8;
    return cls;
}

static pmStatus ensure_host(AddressSpace* a) {
    if (a->host) return pmSuccess;
    Controller& c = ctl();
    const size_t len = a->length ? a->length : 1;
    void* p = nullptr;
    size_t cap = len;
    if (c.has_gpu) {
        cap = pin_class(len);
        {
            std::lock_guard<std::mutex> g(c.pin_mu);
            auto it = c.pin_free.find(cap);
            if (it != c.pin_free.end()) {
                p = it->second;
                c.pin_cached -= cap;
                c.pin_free.erase(it);
            }
        }
        if (!p) {
            const double t0 = now_s();
            if (pmb_host_alloc(&p, cap) != PMB_SUCCESS) return dev_fail(PMB_MEMORY_ERROR, "pinned host allocation");
            c.stats.pin_ns += ns_since(t0);
            c.stats.pin_bytes += cap;
        }
    } else {
        p = malloc(len);
        if (!p) return fail(pmMemoryError, "host allocation of %zu bytes failed", a->length);
    }
    a->host = static_cast<char*>(p);
    a->host_cap = cap;
    return pmSuccess;
}

// Host copy from the pinned cache only (no new allocation): false if none of
// the right class is free.  Used where a pinned allocation would stall the
// stub thread.
static bool host_from_cache(AddressSpace* a) {
    if (a->host) return true;
    Controller& c = ctl();
    if (!c.has_gpu) return false;
    const size_t cap = pin_class(a->length ? a->length : 1);
    std::lock_guard<std::mutex> g(c.pin_mu);
    auto it = c.pin_free.find(cap);
    if (it == c.pin_free.end()) return false;
    a->host = it->second;
    a->host_cap = cap;
    c.pin_cached -= cap;
    c.pin_free.erase(it);
    return true;
}

static void release_host(char* host, size_t cap) {
    Controller& c = ctl();
    if (!c.has_gpu) {
        free(host);
        return;
    }
    {
        std::lock_guard<std::mutex> g(c.pin_mu);
        if (c.pin_cached + cap <= c.pin_limit) {
            c.pin_free.emplace(cap, host);
            c.pin_cached += cap;
            return;
        }
    }
    pmb_host_free(host);
}

static void free_space(AddressSpace* a) {
    if (a->dev) {
        if (a->last_access) pmb_stream_wait_event(ctl().fetch_stream, a->last_access);
        pmb_free_async(a->dev, ctl().fetch_stream);
        ctl().dev_held -= static_cast<int64_t>(a->length);
    }
    if (a->host) release_host(a->host, a->host_cap);
    if (a->last_write) pmb_event_destroy(a->last_write);
    if (a->last_access) pmb_event_destroy(a->last_access);
    delete a;
}

// ---------------------------------------------------------------------------
// subscriptions -> views

static void consolidated(const std::vector<Record>& rs, size_t& lo, size_t& hi) {
    lo = SIZE_MAX;
    hi = 0;
    for (const Record& r : rs) {
        if (!r.count || !r.size) continue;
        lo = std::min(lo, r.lo());
        hi = std::max(hi, r.hi());
    }
    if (lo > hi) lo = hi = 0;
}

static void add_record(RangeSet& s, const Record& r) {
    if (r.contiguous()) {
        s.add(r.offset, r.hi());
        return;
    }
    for (size_t k = 0; k < r.count; ++k) s.add(r.offset + k * r.step, r.offset + k * r.step + r.size);
}

// Union of the byte ranges of `recs`, as sorted disjoint [lo, hi) pieces with
// touching pieces joined.  Records that are rows of one pitch (the 2-D tiles
// of image and matrix subscriptions) are merged band by band: within a band
// of rows the same records are active, so the band is one contiguous piece
// when their columns cover the whole pitch, else the same column pieces
// repeat on every row of the band.  This costs O(records^2 + pieces) instead
// of one ordered-map insertion per row of every record.
static void union_records(const std::vector<const Record*>& recs, std::vector<std::pair<size_t, size_t>>& out) {
    out.clear();
    size_t step = 0;
    bool strided = true;
    for (const Record* r : recs) {
        if (!r->count || !r->size) continue;
        if (r->contiguous() || r->size > r->step) {
            strided = false;
            break;
        }
        if (!step) step = r->step;
        if (r->step != step || (r->offset % step) + r->size > step) {
            strided = false;
            break;
        }
    }
    auto push = [&](size_t lo, size_t hi) {
        if (!out.empty() && out.back().second >= lo) out.back().second = std::max(out.back().second, hi);
        else out.emplace_back(lo, hi);
    };
    if (!strided || !step) {
        RangeSet u;
        for (const Record* r : recs) add_record(u, *r);
        for (auto& kv : u.map()) out.emplace_back(kv.first, kv.second);
        return;
    }
    std::vector<size_t> rows;  // band boundaries
    for (const Record* r : recs) {
        if (!r->count || !r->size) continue;
        rows.push_back(r->offset / step);
        rows.push_back(r->offset / step + r->count);
    }
    std::sort(rows.begin(), rows.end());
    rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
    std::vector<std::pair<size_t, size_t>> cols;
    for (size_t b = 0; b + 1 < rows.size(); ++b) {
        const size_t b0 = rows[b], b1 = rows[b + 1];
        cols.clear();
        for (const Record* r : recs) {
            if (!r->count || !r->size) continue;
            const size_t r0 = r->offset / step;
            if (r0 <= b0 && r0 + r->count >= b1) cols.emplace_back(r->offset % step, r->offset % step + r->size);
        }
        if (cols.empty()) continue;
        std::sort(cols.begin(), cols.end());
        size_t k = 0;  // merge the column pieces in place
        for (size_t i = 1; i < cols.size(); ++i) {
            if (cols[i].first <= cols[k].second) cols[k].second = std::max(cols[k].second, cols[i].second);
            else cols[++k] = cols[i];
        }
        cols.resize(k + 1);
        if (cols.size() == 1 && cols[0].first == 0 && cols[0].second == step) {
            push(b0 * step, b1 * step);
            continue;
        }
        for (size_t row = b0; row < b1; ++row)
            for (auto& c : cols) push(row * step + c.first, row * step + c.second);
    }
}

// Compact layout of one address space for one subtask: the union of its read
// and write ranges, packed back to back in offset order
// (pmSubscriptionManager::GetCompactedSubscription, pmSubscriptionManager.cpp:1978-2030).
struct Compact {
    RangeSet uni;
    std::vector<std::pair<size_t, size_t>> pieces;  // (space offset, length) in packed order
    size_t length = 0;
    size_t offset_of(size_t space_off) const {  // packed offset of a byte inside the union
        size_t covered = 0;
        for (auto& p : pieces) {
            if (space_off >= p.first && space_off < p.first + p.second) return covered + space_off - p.first;
            covered += p.second;
        }
        return covered;
    }
};

static Compact compact_of(const SubtaskMem& m) {
    Compact c;
    for (const Record& r : m.reads) add_record(c.uni, r);
    for (const Record& r : m.writes) add_record(c.uni, r);
    for (auto& kv : c.uni.map()) {
        c.pieces.emplace_back(kv.first, kv.second - kv.first);
        c.length += kv.second - kv.first;
    }
    return c;
}

// ---------------------------------------------------------------------------
// device staging helpers (copy stream unless noted)

// Upload the rows of record `r` that are not yet valid on the device.
static pmStatus upload_record(AddressSpace* a, const Record& r, void* stream) {
    if (!r.count || !r.size) return pmSuccess;
    Controller& c = ctl();
    if (a->dev_valid.covers(r.lo(), r.hi())) return pmSuccess;
    if (!a->host) {  // never written by the host: contents are undefined either way
        add_record(a->dev_valid, r);
        return pmSuccess;
    }
    if (r.contiguous()) {
        std::vector<std::pair<size_t, size_t>> miss;
        a->dev_valid.missing(r.lo(), r.hi(), miss);
        for (auto& m : miss) {
            PMR_DEV(pmb_memcpy_async(a->dev + m.first, a->host + m.first, m.second - m.first, PMB_H2D, stream));
            c.stats.h2d += m.second - m.first;
        }
        a->dev_valid.add(r.lo(), r.hi());
        return pmSuccess;
    }
    // Scattered: 2-D copies over runs of consecutive rows that miss bytes.
    size_t k = 0;
    while (k < r.count) {
        while (k < r.count && a->dev_valid.covers(r.offset + k * r.step, r.offset + k * r.step + r.size)) ++k;
        size_t e = k;
        while (e < r.count && !a->dev_valid.covers(r.offset + e * r.step, r.offset + e * r.step + r.size)) ++e;
        if (e > k) {
            const size_t off = r.offset + k * r.step;
            PMR_DEV(pmb_memcpy2d_async(a->dev + off, r.step, a->host + off, r.step, r.size, e - k, PMB_H2D, stream));
            c.stats.h2d += r.size * (e - k);
        }
        k = e;
    }
    add_record(a->dev_valid, r);
    return pmSuccess;
}

// Copy a record between the mirror and a packed buffer (D2D).
static pmStatus pack_record(AddressSpace* a, const Record& r, const Compact& cp, char* packed, bool to_packed,
                            void* stream) {
    if (!r.count || !r.size) return pmSuccess;
    const size_t poff = cp.offset_of(r.offset);
    if (r.contiguous()) {
        const size_t n = r.hi() - r.lo();
        return to_packed ? (pmb_memcpy_async(packed + poff, a->dev + r.offset, n, PMB_D2D, stream) == PMB_SUCCESS
                                ? pmSuccess
                                : dev_fail(PMB_GRAPHICS_CARD_ERROR, "pack"))
                         : (pmb_memcpy_async(a->dev + r.offset, packed + poff, n, PMB_D2D, stream) == PMB_SUCCESS
                                ? pmSuccess
                                : dev_fail(PMB_GRAPHICS_CARD_ERROR, "unpack"));
    }
    // One 2-D copy when the record's rows sit at a uniform pitch in the packed
    // view (the usual case: rows do not interleave with other records);
    // otherwise one copy per row.
    const size_t ppitch = r.count > 1 ? cp.offset_of(r.offset + r.step) - poff : r.size;
    bool uniform = ppitch >= r.size;
    for (size_t k = 2; uniform && k < r.count; ++k) uniform = cp.offset_of(r.offset + k * r.step) == poff + k * ppitch;
    if (uniform) {
        const int st = to_packed ? pmb_memcpy2d_async(packed + poff, ppitch, a->dev + r.offset, r.step, r.size, r.count,
                                                      PMB_D2D, stream)
                                 : pmb_memcpy2d_async(a->dev + r.offset, r.step, packed + poff, ppitch, r.size, r.count,
                                                      PMB_D2D, stream);
        return st == PMB_SUCCESS ? pmSuccess : dev_fail(st, "compact copy");
    }
    for (size_t k = 0; k < r.count; ++k) {
        const size_t off = r.offset + k * r.step, po = cp.offset_of(off);
        const int st = to_packed ? pmb_memcpy_async(packed + po, a->dev + off, r.size, PMB_D2D, stream)
                                 : pmb_memcpy_async(a->dev + off, packed + po, r.size, PMB_D2D, stream);
        if (st != PMB_SUCCESS) return dev_fail(st, "compact row copy");
    }
    return pmSuccess;
}

// Write the host-stale bytes of [lo, hi) back to the host (synchronous).
static pmStatus fetch_range(AddressSpace* a, size_t lo, size_t hi) {
    Controller& c = ctl();
    std::vector<std::pair<size_t, size_t>> st;
    a->host_stale.present(lo, hi, st);
    if (st.empty()) return pmSuccess;
    const double t0 = now_s();
    const pmStatus hs = ensure_host(a);
    if (hs != pmSuccess) return hs;
    const double t1 = now_s();
    if (a->last_write) PMR_DEV(pmb_event_synchronize(a->last_write));
    const double t2 = now_s();
    for (auto& r : st) {
        PMR_DEV(pmb_memcpy_async(a->host + r.first, a->dev + r.first, r.second - r.first, PMB_D2H, c.fetch_stream));
        c.stats.d2h += r.second - r.first;
    }
    PMR_DEV(pmb_stream_synchronize(c.fetch_stream));
    c.stats.fetch_host_ns += static_cast<unsigned long long>((t1 - t0) * 1e9);
    c.stats.fetch_wait_ns += static_cast<unsigned long long>((t2 - t1) * 1e9);
    c.stats.fetch_copy_ns += ns_since(t2);
    c.stats.fetches++;
    for (auto& r : st) a->host_stale.remove(r.first, r.second);
    return pmSuccess;
}

// Free device mirrors of idle address spaces (least recently used first)
// until `need` more bytes fit in the runtime's device budget (dev_held counts
// the mirrors and reserved subtask memory the runtime holds).
static bool make_room(size_t need, const std::vector<AddressSpace*>& keep) {
    Controller& c = ctl();
    for (;;) {
        if (c.dev_held.load() + static_cast<int64_t>(need) <= c.dev_budget) return true;
        AddressSpace* victim = nullptr;
        {
            std::lock_guard<std::mutex> g(c.mu);
            for (AddressSpace* a : c.spaces) {
                if (!a->dev || a->users > 0) continue;
                if (std::find(keep.begin(), keep.end(), a) != keep.end()) continue;
                if (!victim || a->lru < victim->lru) victim = a;
            }
        }
        if (!victim) return false;
        std::lock_guard<std::mutex> g(victim->mu);
        fetch_range(victim, 0, victim->length);
        if (victim->last_access) pmb_event_synchronize(victim->last_access);
        pmb_free_async(victim->dev, c.fetch_stream);
        pmb_stream_synchronize(c.fetch_stream);
        c.dev_held -= static_cast<int64_t>(victim->length);
        c.stats.evictions++;
        c.stats.evicted_bytes += victim->length;
        victim->dev = nullptr;
        victim->dev_valid.clear();
    }
}

// ---------------------------------------------------------------------------
// task execution: CUDA stub

static pmStatus run_dd(Task* t, const pmDeviceInfo& dev) {
    const pmDataDistributionCallback dd = t->callbacks->cb.dataDistribution;
    t_dd.task = t;
    for (Subtask& s : t->subtasks) {
        if (!dd) continue;
        pmSubtaskInfo si;
        si.subtaskId = s.id;
        si.memCount = static_cast<uint>(t->spaces.size());
        const pmStatus st = dd(t->info, dev, si);
        if (st != pmSuccess) {
            t_dd.task = nullptr;
            return fail(st, "data distribution callback of subtask %lu returned %d", s.id, static_cast<int>(st));
        }
    }
    t_dd.task = nullptr;
    return pmSuccess;
}

// ---------------------------------------------------------------------------
// subtask reduction (pmCallbacks::dataReduction)
//
// Every subtask that writes a writable address space of such a task writes a
// private copy of its subscribed range; when all subtasks have run, the
// copies are folded in subtask-id order and the written bytes committed to
// the address space (pmReducer.cpp:1073-1296 reduces pairs of subtask shadow
// memories over their unified read-write subscription and commits the
// surviving one's write subscription).  Built-in REDUCE_* callbacks fold on
// the device for GPU tasks (one pmb_reduce_elementwise pass); the app's own
// callback runs on the host over host copies, pairwise into the first
// subtask, as the reference calls it.

static bool writable(pmMemType m) { return m != READ_ONLY && m != READ_ONLY_LAZY; }

template <int OP, int TYPE>
static pmStatus builtin_reduction(pmTaskInfo ti, pmDeviceInfo d1, pmSubtaskInfo s1, pmDeviceInfo d2, pmSubtaskInfo s2) {
    return pmReduceSubtasks(ti.taskHandle, d1.deviceHandle, s1.subtaskId, s1.splitInfo, d2.deviceHandle, s2.subtaskId,
                            s2.splitInfo, static_cast<pmReductionOpType>(OP), static_cast<pmReductionDataType>(TYPE));
}

#define PMR_REDUCTION_ROW(op)                                                                              \
    {builtin_reduction<op, 0>, builtin_reduction<op, 1>, builtin_reduction<op, 2>, builtin_reduction<op, 3>, \
     builtin_reduction<op, 4>, builtin_reduction<op, 5>}
// [pmReductionOpType][pmReductionDataType] (pmPublicDefinitions.cpp:749-815)
static const pmDataReductionCallback kBuiltinReduction[10][6] = {
    PMR_REDUCTION_ROW(0), PMR_REDUCTION_ROW(1), PMR_REDUCTION_ROW(2), PMR_REDUCTION_ROW(3), PMR_REDUCTION_ROW(4),
    PMR_REDUCTION_ROW(5), PMR_REDUCTION_ROW(6), PMR_REDUCTION_ROW(7), PMR_REDUCTION_ROW(8), PMR_REDUCTION_ROW(9)};
#undef PMR_REDUCTION_ROW

static bool builtin_of(pmDataReductionCallback cb, int* op, int* type) {
    for (int o = 0; o < 10; ++o)
        for (int d = 0; d < 6; ++d)
            if (kBuiltinReduction[o][d] == cb) {
                *op = o;
                *type = d;
                return true;
            }
    return false;
}

// Bitwise operations on floats and doubles act on the values converted to
// 32- / 64-bit unsigned integers; LOGICAL_XOR is a != b (pmReducer.cpp:408-423, 590-700).
template <typename T, typename B>
static void host_fold(int op, T* a, const T* b, size_t n) {
    switch (op) {
        case REDUCE_ADD: for (size_t i = 0; i < n; ++i) a[i] += b[i]; break;
        case REDUCE_MIN: for (size_t i = 0; i < n; ++i) a[i] = std::min(a[i], b[i]); break;
        case REDUCE_MAX: for (size_t i = 0; i < n; ++i) a[i] = std::max(a[i], b[i]); break;
        case REDUCE_PRODUCT: for (size_t i = 0; i < n; ++i) a[i] *= b[i]; break;
        case REDUCE_LOGICAL_AND: for (size_t i = 0; i < n; ++i) a[i] = (a[i] && b[i]); break;
        case REDUCE_BITWISE_AND: for (size_t i = 0; i < n; ++i) a[i] = static_cast<T>(static_cast<B>(a[i]) & static_cast<B>(b[i])); break;
        case REDUCE_LOGICAL_OR: for (size_t i = 0; i < n; ++i) a[i] = (a[i] || b[i]); break;
        case REDUCE_BITWISE_OR: for (size_t i = 0; i < n; ++i) a[i] = static_cast<T>(static_cast<B>(a[i]) | static_cast<B>(b[i])); break;
        case REDUCE_LOGICAL_XOR: for (size_t i = 0; i < n; ++i) a[i] = (a[i] != b[i]); break;
        default: for (size_t i = 0; i < n; ++i) a[i] = static_cast<T>(static_cast<B>(a[i]) ^ static_cast<B>(b[i])); break;
    }
}

static void host_fold_range(int op, int type, char* a, const char* b, size_t n);

// Large folds are split over the host cores in contiguous element ranges (the
// reference's loops are OpenMP-parallel, pmReducer.cpp:593-700).
static pmStatus host_reduce(int op, int type, void* a, const void* b, size_t bytes) {
    if (op < 0 || op >= MAX_REDUCTION_OP_TYPES) return fail(pmInvalidIndex, "unknown reduction operation %d", op);
    const size_t es = pmb_reduce_element_size(type);
    if (!es) return fail(pmInvalidIndex, "unknown reduction data type %d", type);
    const size_t n = bytes / es;
    const size_t parts = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), n >> 18);
    if (parts <= 1) {
        host_fold_range(op, type, static_cast<char*>(a), static_cast<const char*>(b), n);
        return pmSuccess;
    }
    std::vector<std::thread> pool;
    for (size_t p = 0; p < parts; ++p) {
        const size_t lo = n * p / parts, hi = n * (p + 1) / parts;
        pool.emplace_back(host_fold_range, op, type, static_cast<char*>(a) + lo * es,
                          static_cast<const char*>(b) + lo * es, hi - lo);
    }
    for (auto& th : pool) th.join();
    return pmSuccess;
}

static void host_fold_range(int op, int type, char* a, const char* b, size_t n) {
    switch (type) {
        case REDUCE_INTS: host_fold<int32_t, int32_t>(op, reinterpret_cast<int32_t*>(a), reinterpret_cast<const int32_t*>(b), n); break;
        case REDUCE_UNSIGNED_INTS: host_fold<uint32_t, uint32_t>(op, reinterpret_cast<uint32_t*>(a), reinterpret_cast<const uint32_t*>(b), n); break;
        case REDUCE_LONGS: host_fold<int64_t, int64_t>(op, reinterpret_cast<int64_t*>(a), reinterpret_cast<const int64_t*>(b), n); break;
        case REDUCE_UNSIGNED_LONGS: host_fold<uint64_t, uint64_t>(op, reinterpret_cast<uint64_t*>(a), reinterpret_cast<const uint64_t*>(b), n); break;
        case REDUCE_FLOATS: host_fold<float, uint32_t>(op, reinterpret_cast<float*>(a), reinterpret_cast<const float*>(b), n); break;
        default: host_fold<double, uint64_t>(op, reinterpret_cast<double*>(a), reinterpret_cast<const double*>(b), n); break;
    }
}

// The reducible address spaces of a task and the one range their writing
// subtasks subscribe.  The reference reduces shadow memories positionally
// and asserts equal lengths (pmReducer.cpp:1290); here the ranges must be
// equal, so positions are addresses.
static pmStatus plan_reduction(Task* t) {
    t->reduce.clear();
    t->reduce_op = t->reduce_type = -1;
    const pmDataReductionCallback cb = t->callbacks->cb.dataReduction;
    if (!cb) return pmSuccess;
    builtin_of(cb, &t->reduce_op, &t->reduce_type);
    for (size_t i = 0; i < t->spaces.size(); ++i) {
        if (!writable(t->mem[i].memType)) continue;
        ReduceSpace rs;
        rs.index = i;
        for (const Subtask& s : t->subtasks) {
            const SubtaskMem& m = s.mem[i];
            size_t rlo, rhi, wlo, whi;
            consolidated(m.reads, rlo, rhi);
            consolidated(m.writes, wlo, whi);
            if (whi <= wlo) continue;
            const size_t lo = rhi > rlo ? std::min(rlo, wlo) : wlo, hi = rhi > rlo ? std::max(rhi, whi) : whi;
            if (rs.subtasks.empty()) {
                rs.lo = lo, rs.hi = hi, rs.wlo = wlo, rs.whi = whi;
            } else if (lo != rs.lo || hi != rs.hi || wlo != rs.wlo || whi != rs.whi) {
                return fail(pmInvalidIndex,
                            "reduction over address space %zu: subtasks %zu and %lu subscribe different ranges", i,
                            rs.subtasks.front(), s.id);
            }
            rs.subtasks.push_back(s.id);
        }
        if (rs.subtasks.empty()) continue;
        if (t->mem[i].subscriptionVisibilityType == SUBSCRIPTION_COMPACT)
            return fail(pmInvalidIndex, "reduction over address space %zu needs a natural view", i);
        t->reduce.push_back(rs);
    }
    return pmSuccess;
}

static size_t reduction_bytes(const Task* t) {
    size_t b = 0;
    for (const ReduceSpace& rs : t->reduce) b += (rs.hi - rs.lo) * rs.subtasks.size();
    return b;
}

// memInfo of a reducible address space over a subtask's private copy.
static pmMemInfo shadow_view(const SubtaskMem& m, const ReduceSpace& rs, char* base) {
    pmMemInfo mi;
    mi.visibilityType = SUBSCRIPTION_NATURAL;
    size_t rlo, rhi;
    consolidated(m.reads, rlo, rhi);
    mi.ptr = base;
    mi.readPtr = rhi > rlo ? base + (rlo - rs.lo) : nullptr;
    mi.writePtr = base + (rs.wlo - rs.lo);
    mi.length = rs.hi - rs.lo;
    return mi;
}

// The REDUCTION_TO_REDUCTION scratch buffer of the subtask every other one
// was folded into (pmTask.cpp:1197-1206); the others' were dropped as they
// were folded (pmExecutionStub.cpp:2573).
static void keep_last_reduction_scratch(Task* t, size_t first) {
    auto& m = t->subtasks[first].scratch;
    auto it = m.find(REDUCTION_TO_REDUCTION);
    t->last_reduction_scratch = it != m.end() && !it->second.empty() ? it->second.data() : nullptr;
}

static size_t first_reducing_subtask(const Task* t) {
    size_t first = t->subtasks.size();
    for (const ReduceSpace& rs : t->reduce) first = std::min(first, rs.subtasks.front());
    return first;
}

// Folds the host copies of every reducible address space into the first
// writing subtask's: the built-in operation in id order, or the app's
// callback called pairwise (first, k) as pmReducer calls it.
static pmStatus reduce_host_shadows(Task* t, const pmDeviceInfo& dev) {
    if (t->reduce.empty()) return pmSuccess;
    if (t->reduce_op >= 0) {
        for (const ReduceSpace& rs : t->reduce) {
            std::vector<char>& dst = t->subtasks[rs.subtasks.front()].host_shadow[rs.index];
            for (size_t k = 1; k < rs.subtasks.size(); ++k) {
                const std::vector<char>& src = t->subtasks[rs.subtasks[k]].host_shadow[rs.index];
                const pmStatus st = host_reduce(t->reduce_op, t->reduce_type, dst.data(), src.data(), dst.size());
                if (st != pmSuccess) return st;
            }
        }
        keep_last_reduction_scratch(t, first_reducing_subtask(t));
        return pmSuccess;
    }
    // The app's callback sees every reducible space of both subtasks; the
    // subtasks it folds are those that wrote any of them.
    std::vector<size_t> order;
    for (const ReduceSpace& rs : t->reduce) order.insert(order.end(), rs.subtasks.begin(), rs.subtasks.end());
    std::sort(order.begin(), order.end());
    order.erase(std::unique(order.begin(), order.end()), order.end());
    auto info_of = [&](size_t id) {
        pmSubtaskInfo info;
        info.subtaskId = id;
        info.memCount = static_cast<uint>(t->spaces.size());
        Subtask& s = t->subtasks[id];
        for (const ReduceSpace& rs : t->reduce)
            if (!s.host_shadow[rs.index].empty())
                info.memInfo[rs.index] = shadow_view(s.mem[rs.index], rs, s.host_shadow[rs.index].data());
        return info;
    };
    const pmSubtaskInfo first = info_of(order.front());
    for (size_t k = 1; k < order.size(); ++k) {
        const pmStatus st = t->callbacks->cb.dataReduction(t->info, dev, first, dev, info_of(order[k]));
        if (st != pmSuccess)
            return fail(st, "reduction callback of subtasks %zu and %zu returned %d", order.front(), order[k],
                        static_cast<int>(st));
        t->subtasks[order[k]].scratch.erase(REDUCTION_TO_REDUCTION);
    }
    keep_last_reduction_scratch(t, order.front());
    return pmSuccess;
}

// Commits the first writing subtask's host copy (its write records) to the
// address space's host copy; the device mirror no longer holds those bytes.
static pmStatus commit_host_shadows(Task* t) {
    for (const ReduceSpace& rs : t->reduce) {
        AddressSpace* a = t->spaces[rs.index];
        const Subtask& s0 = t->subtasks[rs.subtasks.front()];
        const std::vector<char>& sh = s0.host_shadow[rs.index];
        std::lock_guard<std::mutex> g(a->mu);
        const pmStatus hs = ensure_host(a);
        if (hs != pmSuccess) return hs;
        for (const Record& r : s0.mem[rs.index].writes)
            for (size_t q = 0; q < std::max<size_t>(r.count, 1); ++q) {
                const size_t off = r.offset + q * r.step;
                memcpy(a->host + off, sh.data() + (off - rs.lo), r.size);
                a->dev_valid.remove(off, off + r.size);
                a->host_stale.remove(off, off + r.size);
            }
    }
    for (Subtask& s : t->subtasks) s.host_shadow.clear();
    return pmSuccess;
}

// GPU tasks: fold the device copies on `stream` (built-in operations) or
// bring them to the host for the app's callback, then free them.
// The device copies of an app's own reduction go to the host for its
// callback.  As the reference does for reduction outputs
// (pmExecutionStub.cpp:3850-3876, pmCudaInterface.cu:380-472), a copy of the
// whole of a single reducible address space larger than the threshold (1 GB,
// CUDA_SENTINEL_COMPRESSION_THRESHOLD; PMB_SENTINEL_THRESHOLD_BYTES
// overrides) is compressed on the device first when fewer than 40 % of its
// elements are non-zero, and expanded on the host.  The app's element type
// is not known here, so the copy is compressed as 32-bit words, which
// restores any data bit for bit.
static pmStatus copy_shadows_to_host(Task* t, void* stream) {
    Controller& c = ctl();
    const char* tv = getenv("PMB_SENTINEL_THRESHOLD_BYTES");
    const size_t threshold = tv ? static_cast<size_t>(atoll(tv)) : (size_t(1) << 30);
    constexpr int kWords = 1;  // REDUCE_UNSIGNED_INTS: 32-bit words
    struct Pending {
        Subtask* s;
        size_t index, len;
        char* buf = nullptr;  // device: compressed form, then scratch
        uint32_t count = 0;
        std::vector<char> packed;
    };
    std::vector<Pending> pend;
    for (const ReduceSpace& rs : t->reduce)
        for (size_t id : rs.subtasks) {
            Subtask& s = t->subtasks[id];
            const size_t len = rs.hi - rs.lo;
            s.host_shadow.resize(t->spaces.size());
            s.host_shadow[rs.index].resize(len);
            const bool whole = t->reduce.size() == 1 && rs.lo == 0 && rs.hi == t->spaces[rs.index]->length;
            if (whole && len > threshold && len % 4 == 0 && len / 4 < (size_t(1) << 32) &&
                (reinterpret_cast<uintptr_t>(s.dev_shadow[rs.index]) & 3) == 0) {
                Pending p;
                p.s = &s;
                p.index = rs.index;
                p.len = len;
                const size_t cap = (pmb_sentinel_capacity_bytes(kWords, len) + 255) & ~size_t(255);
                void* b = nullptr;
                PMR_DEV(pmb_malloc_async(&b, cap + pmb_sentinel_scratch_bytes(kWords, len), stream));
                p.buf = static_cast<char*>(b);
                PMR_DEV(pmb_sentinel_compress(kWords, s.dev_shadow[rs.index], len, p.buf, cap, p.buf + cap,
                                              pmb_sentinel_scratch_bytes(kWords, len), stream));
                pend.push_back(std::move(p));
            } else {
                PMR_DEV(pmb_memcpy_async(s.host_shadow[rs.index].data(), s.dev_shadow[rs.index], len, PMB_D2H, stream));
            }
        }
    for (Pending& p : pend) PMR_DEV(pmb_memcpy_async(&p.count, p.buf, sizeof(uint32_t), PMB_D2H, stream));
    PMR_DEV(pmb_stream_synchronize(stream));
    for (Pending& p : pend) {
        char* host = p.s->host_shadow[p.index].data();
        if (pmb_sentinel_compressed(kWords, p.len, p.count)) {
            const size_t bytes = sizeof(uint32_t) + static_cast<size_t>(p.count) * 8;
            p.packed.resize(bytes);
            PMR_DEV(pmb_memcpy_async(p.packed.data(), p.buf, bytes, PMB_D2H, stream));
            c.stats.sentinel_copies++;
            c.stats.sentinel_bytes += bytes;
        } else {
            PMR_DEV(pmb_memcpy_async(host, p.s->dev_shadow[p.index], p.len, PMB_D2H, stream));
        }
        PMR_DEV(pmb_free_async(p.buf, stream));
    }
    PMR_DEV(pmb_stream_synchronize(stream));
    for (Pending& p : pend)
        if (!p.packed.empty())
            PMR_DEV(pmb_sentinel_expand(kWords, p.packed.data(), p.s->host_shadow[p.index].data(), p.len));
    return pmSuccess;
}

static pmStatus reduce_device_shadows(Task* t, void* stream) {
    if (t->reduce.empty()) return pmSuccess;
    if (t->reduce_op >= 0) {
        const size_t es = pmb_reduce_element_size(t->reduce_type);
        for (const ReduceSpace& rs : t->reduce) {
            AddressSpace* a = t->spaces[rs.index];
            const Subtask& s0 = t->subtasks[rs.subtasks.front()];
            const SubtaskMem& m0 = s0.mem[rs.index];
            std::vector<const void*> srcs;
            for (size_t id : rs.subtasks) srcs.push_back(t->subtasks[id].dev_shadow[rs.index]);
            RangeSet w;
            for (const Record& r : m0.writes) add_record(w, r);
            std::lock_guard<std::mutex> g(a->mu);
            // Contiguous, element-aligned writes fold straight into the mirror;
            // otherwise into the first copy, whose written records are then copied.
            if (w.covers(rs.wlo, rs.whi) && rs.wlo % es == 0 && (rs.wlo - rs.lo) % es == 0 &&
                (rs.whi - rs.wlo) % es == 0) {
                for (const void*& p : srcs) p = static_cast<const char*>(p) + (rs.wlo - rs.lo);
                PMR_DEV(pmb_reduce_elementwise(t->reduce_op, t->reduce_type, a->dev + rs.wlo, srcs.data(),
                                               static_cast<int>(srcs.size()), (rs.whi - rs.wlo) / es, 1, stream));
            } else {
                char* s0p = s0.dev_shadow[rs.index];
                if (srcs.size() > 1)
                    PMR_DEV(pmb_reduce_elementwise(t->reduce_op, t->reduce_type, s0p, srcs.data() + 1,
                                                   static_cast<int>(srcs.size() - 1), (rs.hi - rs.lo) / es, 0, stream));
                for (auto& piece : w.map())
                    PMR_DEV(pmb_memcpy_async(a->dev + piece.first, s0p + (piece.first - rs.lo),
                                             piece.second - piece.first, PMB_D2D, stream));
            }
            for (const Record& r : m0.writes) {
                add_record(a->dev_valid, r);
                add_record(a->host_stale, r);
            }
        }
        keep_last_reduction_scratch(t, first_reducing_subtask(t));
    } else {
        PMR_DEV(pmb_stream_synchronize(stream));
        const pmStatus cs = copy_shadows_to_host(t, stream);
        if (cs != pmSuccess) return cs;
        pmStatus st = reduce_host_shadows(t, ctl().gpu_info);
        if (st == pmSuccess) st = commit_host_shadows(t);
        if (st != pmSuccess) return st;
    }
    for (Subtask& s : t->subtasks)
        for (char*& p : s.dev_shadow)
            if (p) {
                PMR_DEV(pmb_free_async(p, stream));
                p = nullptr;
            }
    return pmSuccess;
}

// ---------------------------------------------------------------------------
// ordered redistribution (pmCallbacks::dataRedistribution, pmRedistributeData)
//
// After a task's subtasks have run, the app's redistribution callback is
// called for each subtask in id order (on the host) and names byte ranges of
// an address space with an order number.  The address space is then rebuilt
// with every order's ranges back to back, orders ascending, ranges within an
// order by subtask id then call order, the rest zero
// (pmRedistributor.cpp:88-121 sums each order's bytes, 123-145 assigns
// running offsets, 240-283 copies the ranges into a new address space that
// replaces the task's, pmTask.cpp:834-856).  A GPU task moves the bytes on
// the device into a new mirror, all ranges in one gather launch.

struct RedistCopy {
    size_t src, dst, len;
};

// Copies and metadata of address space i; fails when the ranges add up to
// more than the address space.
static pmStatus redist_plan(Task* t, size_t i, std::vector<RedistCopy>& copies) {
    std::vector<RedistRecord>& rs = t->redist[i];
    std::sort(rs.begin(), rs.end(), [](const RedistRecord& a, const RedistRecord& b) {
        return a.order != b.order ? a.order < b.order : (a.subtask != b.subtask ? a.subtask < b.subtask : a.seq < b.seq);
    });
    copies.clear();
    t->redist_meta.resize(t->spaces.size());
    std::vector<pmRedistributionMetadata>& meta = t->redist_meta[i];
    meta.clear();
    size_t run = 0;
    for (const RedistRecord& r : rs) {
        if (run + r.length > t->spaces[i]->length)
            return fail(pmInvalidIndex, "redistribution of address space %zu: %zu bytes beyond its %zu", i,
                        run + r.length, t->spaces[i]->length);
        if (!copies.empty() && copies.back().src + copies.back().len == r.offset)
            copies.back().len += r.length;  // continues the previous range in both places: one copy
        else
            copies.push_back({r.offset, run, r.length});
        if (meta.empty() || meta.back().order != r.order) meta.emplace_back(r.order, 0u);
        meta.back().count += static_cast<uint>(r.length);
        run += r.length;
    }
    return pmSuccess;
}

static pmStatus run_redistribution_callbacks(Task* t, const pmDeviceInfo& dev) {
    const pmDataRedistributionCallback cb = t->callbacks->cb.dataRedistribution;
    {
        std::lock_guard<std::mutex> g(t->redist_mu);
        t->redist.assign(t->spaces.size(), {});
        t->redist_open = true;
    }
    pmStatus st = pmSuccess;
    for (Subtask& s : t->subtasks) {
        pmSubtaskInfo info;
        info.subtaskId = s.id;
        info.memCount = static_cast<uint>(t->spaces.size());
        st = cb(t->info, dev, info);
        if (st != pmSuccess) {
            st = fail(st, "redistribution callback of subtask %lu returned %d", s.id, static_cast<int>(st));
            break;
        }
    }
    std::lock_guard<std::mutex> g(t->redist_mu);
    t->redist_open = false;
    return st;
}

// GPU task: after its work (the callbacks read SUBTASK_TO_POST_SUBTASK
// scratch buffers, copied back on the task's streams), each redistributed
// address space gets a new zeroed mirror filled by device copies on `stream`.
static pmStatus redistribute_device(Task* t, void* stream) {
    Controller& c = ctl();
    PMR_DEV(pmb_stream_synchronize(stream));
    pmStatus st = run_redistribution_callbacks(t, c.gpu_info);
    if (st != pmSuccess) return st;
    std::vector<RedistCopy> copies;
    for (size_t i = 0; i < t->spaces.size(); ++i) {
        if (t->redist[i].empty()) continue;
        st = redist_plan(t, i, copies);
        if (st != pmSuccess) return st;
        AddressSpace* a = t->spaces[i];
        std::lock_guard<std::mutex> g(a->mu);
        for (const RedistCopy& k : copies) {  // source bytes the device does not hold come from the host
            Record r;
            r.offset = k.src, r.size = k.len, r.step = k.len, r.count = 1;
            st = upload_record(a, r, stream);
            if (st != pmSuccess) return st;
        }
        void* nd = nullptr;
        PMR_DEV(pmb_malloc_async(&nd, a->length ? a->length : 1, stream));
        PMR_DEV(pmb_memset_async(nd, 0, a->length, stream));
        if (copies.size() <= 4) {
            for (const RedistCopy& k : copies)
                PMR_DEV(pmb_memcpy_async(static_cast<char*>(nd) + k.dst, a->dev + k.src, k.len, PMB_D2D, stream));
        } else {  // all ranges in one launch, the range table staged on the device
            std::vector<pmb_copy_range> table(copies.size());
            for (size_t k = 0; k < copies.size(); ++k) table[k] = {copies[k].src, copies[k].dst, copies[k].len};
            void* dt = nullptr;
            const size_t tb = table.size() * sizeof(pmb_copy_range);
            PMR_DEV(pmb_malloc_async(&dt, tb, stream));
            PMR_DEV(pmb_memcpy_async(dt, table.data(), tb, PMB_H2D, stream));
            PMR_DEV(pmb_copy_ranges(nd, a->dev, static_cast<const pmb_copy_range*>(dt), static_cast<int>(table.size()),
                                    stream));
            PMR_DEV(pmb_stream_synchronize(stream));  // the table is a host vector (pageable copy)
            PMR_DEV(pmb_free_async(dt, stream));
        }
        PMR_DEV(pmb_free_async(a->dev, stream));
        a->dev = static_cast<char*>(nd);
        a->dev_valid.clear();
        a->dev_valid.add(0, a->length);
        a->host_stale.clear();
        a->host_stale.add(0, a->length);
    }
    return pmSuccess;
}

// CPU task: the same permutation of the host copy.
static pmStatus redistribute_host(Task* t) {
    pmStatus st = run_redistribution_callbacks(t, ctl().cpu_info);
    if (st != pmSuccess) return st;
    std::vector<RedistCopy> copies;
    for (size_t i = 0; i < t->spaces.size(); ++i) {
        if (t->redist[i].empty()) continue;
        st = redist_plan(t, i, copies);
        if (st != pmSuccess) return st;
        AddressSpace* a = t->spaces[i];
        std::lock_guard<std::mutex> g(a->mu);
        const std::vector<char> old(a->host, a->host + a->length);
        memset(a->host, 0, a->length);
        for (const RedistCopy& k : copies) memcpy(a->host + k.dst, old.data() + k.src, k.len);
        a->dev_valid.clear();
        a->host_stale.clear();
    }
    return pmSuccess;
}

// Admission by free device memory: the task's missing mirrors and reserved
// subtask memory must fit beside the reserve, after idle mirrors are evicted.
static bool admit(Task* t, size_t* need_out) {
    size_t need = 0;
    for (AddressSpace* a : t->spaces)
        if (!a->dev) need += a->length;
    for (Subtask& s : t->subtasks) need += s.reserved;
    need += reduction_bytes(t);
    *need_out = need;
    return need == 0 || make_room(need, t->spaces);
}

// Upload what subtasks [g0, g1) of a batched task read and the device lacks.
// Their read records are merged first: neighbouring tiles' rows join into
// long contiguous copies (one per run of full rows for a row of image tiles)
// instead of one narrow 2-D copy per subtask; when merging would not reduce
// the number of copies, each record is uploaded on its own.
static pmStatus upload_group(Task* t, size_t g0, size_t g1, void* stream) {
    Controller& c = ctl();
    std::vector<const Record*> recs;
    std::vector<std::pair<size_t, size_t>> need;
    for (size_t i = 0; i < t->spaces.size(); ++i) {
        AddressSpace* a = t->spaces[i];
        std::lock_guard<std::mutex> g(a->mu);
        recs.clear();
        for (size_t si = g0; si < g1; ++si)
            for (const Record& r : t->subtasks[si].mem[i].reads)
                if (r.count && r.size) recs.push_back(&r);
        if (recs.empty()) continue;
        union_records(recs, need);
        if (need.size() > recs.size()) {
            for (const Record* r : recs) {
                const pmStatus st = upload_record(a, *r, stream);
                if (st != pmSuccess) return st;
            }
            continue;
        }
        for (auto& kv : need) {
            if (a->host) {  // never written by the host: contents are undefined either way
                std::vector<std::pair<size_t, size_t>> miss;
                a->dev_valid.missing(kv.first, kv.second, miss);
                for (auto& m : miss) {
                    PMR_DEV(pmb_memcpy_async(a->dev + m.first, a->host + m.first, m.second - m.first, PMB_H2D, stream));
                    c.stats.h2d += m.second - m.first;
                }
            }
            a->dev_valid.add(kv.first, kv.second);
        }
    }
    return pmSuccess;
}

// Record what subtasks [g0, g1) of a batched task wrote (valid on the device,
// newer than the host) and, when results go to the host at task end (cache
// disabled, or eager write-back), copy those bytes back on `stream` right
// after the group's launch: a group's results then cross to the host while
// later groups compute.  Fragmented write sets are left to the task-end
// write-back.
static pmStatus writeback_group(Task* t, size_t g0, size_t g1, bool write_through, void* stream) {
    Controller& c = ctl();
    std::vector<const Record*> recs;
    std::vector<std::pair<size_t, size_t>> done;
    for (size_t i = 0; i < t->spaces.size(); ++i) {
        if (!writable(t->mem[i].memType)) continue;
        AddressSpace* a = t->spaces[i];
        std::lock_guard<std::mutex> g(a->mu);
        recs.clear();
        for (size_t si = g0; si < g1; ++si)
            for (const Record& r : t->subtasks[si].mem[i].writes)
                if (r.count && r.size) recs.push_back(&r);
        if (recs.empty()) continue;
        union_records(recs, done);
        // Mark the group's results valid on the device and newer than the host.
        for (auto& kv : done) {
            a->dev_valid.add(kv.first, kv.second);
            a->host_stale.add(kv.first, kv.second);
        }
        if (!write_through && !c.eager_writeback) continue;
        if (done.size() > std::max<size_t>(recs.size(), 16)) continue;  // fragmented: left to the task-end write-back
        if (write_through) {
            const pmStatus hs = ensure_host(a);
            if (hs != pmSuccess) return hs;
        } else if (!host_from_cache(a)) {
            continue;  // no pinned buffer at hand: pmFetchMemory copies it back later
        }
        for (auto& kv : done) {
            PMR_DEV(pmb_memcpy_async(a->host + kv.first, a->dev + kv.first, kv.second - kv.first, PMB_D2H, stream));
            c.stats.d2h += kv.second - kv.first;
            a->host_stale.remove(kv.first, kv.second);
        }
    }
    return pmSuccess;
}

static pmStatus stage_and_launch_gpu(Task* t) {
    Controller& c = ctl();
    const pmCallbacks& cb = t->callbacks->cb;
    const size_t ns = t->spaces.size();
    const bool write_through = !t->details.cudaCacheEnabled || env_flag("PMLIB_DISABLE_CUDA_CACHE");

    // Views: OPTIMAL is NATURAL here -- every address space has a resident
    // mirror, so natural views need no packing copies.
    t->views.resize(ns);
    for (size_t i = 0; i < ns; ++i)
        t->views[i] = t->mem[i].subscriptionVisibilityType == SUBSCRIPTION_COMPACT ? SUBSCRIPTION_COMPACT
                                                                                  : SUBSCRIPTION_NATURAL;

    // Device mirrors (admission by free device memory happened in admit()).
    for (AddressSpace* a : t->spaces) {
        std::lock_guard<std::mutex> g(a->mu);
        if (!a->dev) {
            void* p = nullptr;  // stream-ordered: no device-wide synchronisation
            PMR_DEV(pmb_malloc_async(&p, a->length ? a->length : 1, c.copy_stream));
            a->dev = static_cast<char*>(p);
            c.dev_held += static_cast<int64_t>(a->length);
        }
        a->lru = ++c.lru;
    }

    // Dependencies on earlier tasks: read-after-write, write-after-access.
    for (size_t i = 0; i < ns; ++i) {
        AddressSpace* a = t->spaces[i];
        const bool writes = t->mem[i].memType != READ_ONLY && t->mem[i].memType != READ_ONLY_LAZY;
        void* ev = writes ? a->last_access : a->last_write;
        if (ev) PMR_DEV(pmb_stream_wait_event(c.copy_stream, ev));
    }

    // Task configuration on the device for subtask_gpu_cuda kernels.
    t->dev_info = t->info;
    if (cb.subtask_gpu_cuda && !t->conf.empty()) {
        PMR_DEV(pmb_malloc_async(&t->dev_conf, t->conf.size(), c.copy_stream));
        PMR_DEV(pmb_memcpy_async(t->dev_conf, t->conf.data(), t->conf.size(), PMB_H2D, c.copy_stream));
        t->dev_info.taskConf = t->dev_conf;
    }

    BatchFn batch = nullptr;
    size_t groups = c.batch_groups;
    if (cb.subtask_gpu_custom && !c.batch_off) {
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.batch.find(reinterpret_cast<void*>(cb.subtask_gpu_custom));
        if (it != c.batch.end()) {
            batch = it->second.fn;
            if (it->second.groups) groups = it->second.groups;
        }
        for (size_t i = 0; i < ns && batch; ++i)
            if (t->views[i] != SUBSCRIPTION_NATURAL) batch = nullptr;
        for (Subtask& s : t->subtasks)
            if (s.reserved || !s.scratch.empty()) batch = nullptr;
        if (!t->reduce.empty()) batch = nullptr;  // each subtask writes its own copy
    }
    std::vector<const ReduceSpace*> reducible(ns, nullptr);
    for (const ReduceSpace& rs : t->reduce) reducible[rs.index] = &rs;

    std::vector<void*> events;
    auto new_event = [&]() -> void* {
        void* e = nullptr;
        if (pmb_event_create(&e, 0) != PMB_SUCCESS) return nullptr;
        events.push_back(e);
        return e;
    };

    std::vector<pmSubtaskInfo> infos(t->subtasks.size());
    std::vector<bool> used_stream(c.streams.size(), false);
    // A batched task runs as up to c.batch_groups launches over consecutive
    // subtasks; each launches once its own group is staged.
    std::vector<size_t> group_begin;  // first subtask of each group, then the subtask count
    std::vector<void*> group_staged;
    if (batch) {
        const size_t nsub = t->subtasks.size();
        const size_t per = (nsub + std::max<size_t>(groups, 1) - 1) / std::max<size_t>(groups, 1);
        for (size_t g0 = 0; g0 < nsub; g0 += std::max<size_t>(per, 1)) group_begin.push_back(g0);
        group_begin.push_back(nsub);
    }
    size_t group = 0;
    for (size_t si = 0; si < t->subtasks.size(); ++si) {
        Subtask& s = t->subtasks[si];
        pmSubtaskInfo& info = infos[si];
        info.subtaskId = s.id;
        info.memCount = static_cast<uint>(ns);
        s.dev_compact.assign(ns, nullptr);
        s.dev_shadow.assign(ns, nullptr);
        std::vector<Compact> compacts(ns);
        // ---- stage (copy stream) ----
        if (batch && si == group_begin[group]) {
            const pmStatus st = upload_group(t, si, group_begin[group + 1], c.copy_stream);
            if (st != pmSuccess) return st;
        }
        for (size_t i = 0; i < ns; ++i) {
            AddressSpace* a = t->spaces[i];
            const SubtaskMem& m = s.mem[i];
            std::lock_guard<std::mutex> g(a->mu);
            for (const Record& r : m.reads) {
                if (batch) break;  // staged with its group
                const pmStatus st = upload_record(a, r, c.copy_stream);
                if (st != pmSuccess) return st;
            }
            pmMemInfo mi;
            mi.visibilityType = t->views[i];
            size_t rlo, rhi, wlo, whi;
            consolidated(m.reads, rlo, rhi);
            consolidated(m.writes, wlo, whi);
            const bool has_r = rhi > rlo, has_w = whi > wlo;
            if (!has_r && !has_w) {
                info.memInfo[i] = mi;
                continue;
            }
            if (has_w && reducible[i]) {
                // private copy of the subscribed range, holding the read bytes
                const ReduceSpace& rs = *reducible[i];
                void* p = nullptr;
                PMR_DEV(pmb_malloc_async(&p, rs.hi - rs.lo, c.copy_stream));
                s.dev_shadow[i] = static_cast<char*>(p);
                c.dev_held += static_cast<int64_t>(rs.hi - rs.lo);  // returned when the task finishes
                t->reserved_held += rs.hi - rs.lo;
                if (has_r) PMR_DEV(pmb_memcpy_async(p, a->dev + rs.lo, rs.hi - rs.lo, PMB_D2D, c.copy_stream));
                info.memInfo[i] = shadow_view(m, rs, s.dev_shadow[i]);
                continue;
            }
            if (t->views[i] == SUBSCRIPTION_NATURAL) {
                const size_t lo = has_r && has_w ? std::min(rlo, wlo) : (has_r ? rlo : wlo);
                const size_t hi = has_r && has_w ? std::max(rhi, whi) : (has_r ? rhi : whi);
                mi.ptr = a->dev + lo;
                mi.readPtr = has_r ? a->dev + rlo : nullptr;
                mi.writePtr = has_w ? a->dev + wlo : nullptr;
                mi.length = hi - lo;
            } else {
                compacts[i] = compact_of(m);
                PMR_DEV(pmb_malloc_async(&s.dev_compact[i], compacts[i].length, c.copy_stream));
                char* packed = static_cast<char*>(s.dev_compact[i]);
                for (const Record& r : m.reads) {
                    const pmStatus st = pack_record(a, r, compacts[i], packed, true, c.copy_stream);
                    if (st != pmSuccess) return st;
                }
                mi.ptr = packed;
                mi.readPtr = has_r ? packed + compacts[i].offset_of(m.reads.front().offset) : nullptr;
                mi.writePtr = has_w ? packed + compacts[i].offset_of(m.writes.front().offset) : nullptr;
                mi.length = compacts[i].length;
            }
            info.memInfo[i] = mi;
        }
        if (batch) {  // launched per group below
            if (si + 1 == group_begin[group + 1]) {
                void* staged = new_event();
                if (!staged) return fail(pmGraphicsCardError, "event creation failed: %s", pmb_last_error());
                PMR_DEV(pmb_event_record(staged, c.copy_stream));
                group_staged.push_back(staged);
                ++group;
            }
            continue;
        }
        void* staged = new_event();
        if (!staged) return fail(pmGraphicsCardError, "event creation failed: %s", pmb_last_error());
        PMR_DEV(pmb_event_record(staged, c.copy_stream));

        // ---- launch (compute stream) ----
        const size_t sidx = c.next_stream++ % c.streams.size();
        void* stream = c.streams[sidx];
        used_stream[sidx] = true;
        PMR_DEV(pmb_stream_wait_event(stream, staged));
        if (s.reserved) {
            PMR_DEV(pmb_malloc_async(&s.dev_reserved, s.reserved, stream));
            c.dev_held += static_cast<int64_t>(s.reserved);  // returned when the task finishes
            t->reserved_held += s.reserved;
            info.gpuContext.reservedGlobalMem = s.dev_reserved;
        }
        auto sc = s.scratch.find(PRE_SUBTASK_TO_SUBTASK);
        if (sc == s.scratch.end()) sc = s.scratch.find(PRE_SUBTASK_TO_POST_SUBTASK);
        if (sc == s.scratch.end()) sc = s.scratch.find(SUBTASK_TO_POST_SUBTASK);
        if (sc != s.scratch.end() && !sc->second.empty()) {
            PMR_DEV(pmb_malloc_async(&s.dev_scratch, sc->second.size(), stream));
            if (sc->first != SUBTASK_TO_POST_SUBTASK)
                PMR_DEV(pmb_memcpy_async(s.dev_scratch, sc->second.data(), sc->second.size(), PMB_H2D, stream));
            info.gpuContext.scratchBuffer = s.dev_scratch;
        }
        s.info = info;
        pmStatus st = pmSuccess;
        if (cb.subtask_gpu_custom) {
            const double tcb = now_s();
            st = cb.subtask_gpu_custom(t->info, c.gpu_info, info, stream);
            c.stats.callback_ns += ns_since(tcb);
        } else {
            const pmCudaLaunchConf lc = s.has_conf ? s.conf : pmCudaLaunchConf();
            pmTaskInfo ti = t->dev_info;
            void* dinfo = c.dev_device_info;
            pmSubtaskInfo sinfo = info;
            void* dstat = c.dev_status;
            void* args[4] = {&ti, &dinfo, &sinfo, &dstat};
            const int ls = pmb_launch_kernel(reinterpret_cast<const void*>(cb.subtask_gpu_cuda), lc.blocksX, lc.blocksY,
                                             lc.blocksZ, lc.threadsX, lc.threadsY, lc.threadsZ, lc.sharedMem, args,
                                             stream);
            if (ls != PMB_SUCCESS) return dev_fail(ls, "subtask kernel launch");
        }
        if (st != pmSuccess) return fail(st, "GPU callback of subtask %lu returned %d", s.id, static_cast<int>(st));
        c.stats.gpu_subtasks++;
        // ---- results (compute stream) ----
        for (size_t i = 0; i < ns; ++i) {
            AddressSpace* a = t->spaces[i];
            const SubtaskMem& m = s.mem[i];
            if (m.writes.empty() || s.dev_shadow[i]) continue;  // private copies are folded after the join
            std::lock_guard<std::mutex> g(a->mu);
            if (t->views[i] == SUBSCRIPTION_COMPACT) {
                for (const Record& r : m.writes) {
                    const pmStatus ps = pack_record(a, r, compacts[i], static_cast<char*>(s.dev_compact[i]), false, stream);
                    if (ps != pmSuccess) return ps;
                }
            }
            for (const Record& r : m.writes) {
                add_record(a->dev_valid, r);
                add_record(a->host_stale, r);
            }
        }
        if (s.dev_scratch && (sc->first == SUBTASK_TO_POST_SUBTASK || sc->first == PRE_SUBTASK_TO_POST_SUBTASK))
            PMR_DEV(pmb_memcpy_async(sc->second.data(), s.dev_scratch, sc->second.size(), PMB_D2H, stream));
        for (size_t i = 0; i < ns; ++i)
            if (s.dev_compact[i]) PMR_DEV(pmb_free_async(s.dev_compact[i], stream));
        if (s.dev_reserved) PMR_DEV(pmb_free_async(s.dev_reserved, stream));
        if (s.dev_scratch) PMR_DEV(pmb_free_async(s.dev_scratch, stream));
    }

    for (size_t gi = 0; batch && gi + 1 < group_begin.size(); ++gi) {
        const size_t g0 = group_begin[gi], g1 = group_begin[gi + 1];
        const size_t sidx = c.next_stream++ % c.streams.size();
        void* stream = c.streams[sidx];
        used_stream[sidx] = true;
        PMR_DEV(pmb_stream_wait_event(stream, group_staged[gi]));  // the group's uploads are done
        const double tcb = now_s();
        const pmStatus st = batch(&t->info, &c.gpu_info, infos.data() + g0, g1 - g0, stream);
        c.stats.callback_ns += ns_since(tcb);
        if (st != pmSuccess) return fail(st, "batched GPU callback returned %d", static_cast<int>(st));
        c.stats.batched++;
        c.stats.gpu_subtasks += g1 - g0;
        for (size_t si = g0; si < g1; ++si) t->subtasks[si].info = infos[si];
        const pmStatus ws = writeback_group(t, g0, g1, write_through, stream);
        if (ws != pmSuccess) return ws;
    }

    // ---- join the task's streams into its completion event ----
    // The join point is the last compute stream the task used (the copy stream
    // for a task without launches), so a task's completion waits only for its
    // own work, never for unrelated tasks on other streams.
    void* join = c.copy_stream;
    for (size_t k = 0; k < c.streams.size(); ++k)
        if (used_stream[k]) join = c.streams[k];
    auto join_on = [&](void* from) -> pmStatus {
        if (from == join) return pmSuccess;
        void* e = new_event();
        if (!e) return fail(pmGraphicsCardError, "event creation failed");
        PMR_DEV(pmb_event_record(e, from));
        PMR_DEV(pmb_stream_wait_event(join, e));
        return pmSuccess;
    };
    {
        pmStatus js = join_on(c.copy_stream);
        for (size_t k = 0; k < c.streams.size() && js == pmSuccess; ++k)
            if (used_stream[k]) js = join_on(c.streams[k]);
        if (js != pmSuccess) return js;
    }
    {
        pmStatus rs = reduce_device_shadows(t, join);
        if (rs == pmSuccess && cb.dataRedistribution) rs = redistribute_device(t, join);
        if (rs != pmSuccess) return rs;
    }
    // Write-back at task end: all stale bytes with the cache disabled (the
    // mirrors are then dropped); with eager write-back (PMB_EAGER_WRITEBACK=1)
    // the bytes of the address spaces this task writes, on the task's own
    // stream so the copies overlap other tasks' kernels, keeping the mirrors.
    if (write_through || c.eager_writeback) {
        for (size_t i = 0; i < ns; ++i) {
            AddressSpace* a = t->spaces[i];
            const bool writes = t->mem[i].memType != READ_ONLY && t->mem[i].memType != READ_ONLY_LAZY;
            if (!write_through && !writes) continue;
            std::lock_guard<std::mutex> g(a->mu);
            std::vector<std::pair<size_t, size_t>> st;
            a->host_stale.present(0, a->length, st);
            if (!st.empty()) {
                if (write_through) {
                    const pmStatus hs = ensure_host(a);
                    if (hs != pmSuccess) return hs;
                } else if (!host_from_cache(a)) {
                    continue;  // no pinned buffer at hand: pmFetchMemory copies it back later
                }
            }
            for (auto& r : st) {
                PMR_DEV(pmb_memcpy_async(a->host + r.first, a->dev + r.first, r.second - r.first, PMB_D2H, join));
                c.stats.d2h += r.second - r.first;
            }
            a->host_stale.clear();
        }
    }
    if (t->dev_conf) PMR_DEV(pmb_free_async(t->dev_conf, join));
    t->dev_conf = nullptr;
    PMR_DEV(pmb_event_record(t->done_event, join));
    for (size_t i = 0; i < ns; ++i) {
        AddressSpace* a = t->spaces[i];
        std::lock_guard<std::mutex> g(a->mu);
        if (!a->last_access) PMR_DEV(pmb_event_create(&a->last_access, 0));
        PMR_DEV(pmb_event_record(a->last_access, join));
        const bool writes = t->mem[i].memType != READ_ONLY && t->mem[i].memType != READ_ONLY_LAZY;
        if (writes) {
            if (!a->last_write) PMR_DEV(pmb_event_create(&a->last_write, 0));
            PMR_DEV(pmb_event_record(a->last_write, join));
        }
        if (write_through) a->dev_valid.clear();
    }
    // Events may be destroyed once recorded: CUDA keeps recorded work alive.
    for (void* e : events) pmb_event_destroy(e);
    return pmSuccess;
}

// CPU execution (tasks whose callbacks have no GPU subtask function): NATURAL
// views of the host copies, subtasks spread over the host cores.
static pmStatus run_cpu_task(Task* t) {
    const size_t ns = t->spaces.size();
    if (!t->callbacks->cb.subtask_cpu) return pmSuccess;  // placement-only task
    for (size_t i = 0; i < ns; ++i) {
        AddressSpace* a = t->spaces[i];
        std::lock_guard<std::mutex> g(a->mu);
        pmStatus st = ensure_host(a);
        if (st != pmSuccess) return st;
        st = fetch_range(a, 0, a->length);
        if (st != pmSuccess) return st;
    }
    // Private copies of the reducible address spaces, holding the bytes of
    // the address space (pmSubscriptionManager.cpp:1530-1537 fills them from
    // the read subscriptions).
    std::vector<const ReduceSpace*> reducible(ns, nullptr);
    for (const ReduceSpace& rs : t->reduce) {
        reducible[rs.index] = &rs;
        const char* src = t->spaces[rs.index]->host;
        for (size_t id : rs.subtasks) {
            Subtask& s = t->subtasks[id];
            s.host_shadow.resize(ns);
            s.host_shadow[rs.index].assign(src + rs.lo, src + rs.hi);
        }
    }
    const unsigned nthreads = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(),
                                                              static_cast<unsigned>(t->subtasks.size())));
    std::atomic<size_t> next(0);
    std::atomic<int> err(pmSuccess);
    auto worker = [&]() {
        for (;;) {
            const size_t k = next.fetch_add(1);
            if (k >= t->subtasks.size() || err.load() != pmSuccess) break;
            if (t->deadline > 0 && now_s() > t->deadline) {
                err.store(pmStatusUnavailable);
                break;
            }
            Subtask& s = t->subtasks[k];
            pmSubtaskInfo info;
            info.subtaskId = s.id;
            info.memCount = static_cast<uint>(ns);
            std::vector<std::vector<char>> packed(ns);
            std::vector<Compact> compacts(ns);
            for (size_t i = 0; i < ns; ++i) {
                AddressSpace* a = t->spaces[i];
                const SubtaskMem& m = s.mem[i];
                size_t rlo, rhi, wlo, whi;
                consolidated(m.reads, rlo, rhi);
                consolidated(m.writes, wlo, whi);
                const bool has_r = rhi > rlo, has_w = whi > wlo;
                pmMemInfo mi;
                mi.visibilityType = t->mem[i].subscriptionVisibilityType == SUBSCRIPTION_COMPACT ? SUBSCRIPTION_COMPACT
                                                                                               : SUBSCRIPTION_NATURAL;
                if (has_w && reducible[i]) {
                    info.memInfo[i] = shadow_view(m, *reducible[i], s.host_shadow[i].data());
                    continue;
                }
                if (has_r || has_w) {
                    if (mi.visibilityType == SUBSCRIPTION_NATURAL) {
                        const size_t lo = has_r && has_w ? std::min(rlo, wlo) : (has_r ? rlo : wlo);
                        const size_t hi = has_r && has_w ? std::max(rhi, whi) : (has_r ? rhi : whi);
                        mi.ptr = a->host + lo;
                        mi.readPtr = has_r ? a->host + rlo : nullptr;
                        mi.writePtr = has_w ? a->host + wlo : nullptr;
                        mi.length = hi - lo;
                    } else {
                        compacts[i] = compact_of(m);
                        packed[i].assign(compacts[i].length, 0);
                        for (auto& pc : compacts[i].pieces)
                            memcpy(packed[i].data() + compacts[i].offset_of(pc.first), a->host + pc.first, pc.second);
                        mi.ptr = packed[i].data();
                        mi.readPtr = has_r ? packed[i].data() + compacts[i].offset_of(m.reads.front().offset) : nullptr;
                        mi.writePtr = has_w ? packed[i].data() + compacts[i].offset_of(m.writes.front().offset) : nullptr;
                        mi.length = compacts[i].length;
                    }
                }
                info.memInfo[i] = mi;
            }
            const pmStatus st = t->callbacks->cb.subtask_cpu(t->info, ctl().cpu_info, info);
            if (st != pmSuccess) {
                err.store(st);
                break;
            }
            for (size_t i = 0; i < ns; ++i) {
                if (!packed[i].empty())
                    for (const Record& r : s.mem[i].writes)
                        for (size_t q = 0; q < std::max<size_t>(r.count, 1); ++q) {
                            const size_t off = r.offset + q * r.step;
                            memcpy(t->spaces[i]->host + off, packed[i].data() + compacts[i].offset_of(off), r.size);
                        }
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned k = 1; k < nthreads; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (err.load() == pmSuccess && !t->reduce.empty()) {
        pmStatus rs = reduce_host_shadows(t, ctl().cpu_info);
        if (rs == pmSuccess) rs = commit_host_shadows(t);
        if (rs != pmSuccess) return rs;
    }
    if (err.load() == pmSuccess && t->callbacks->cb.dataRedistribution) {
        const pmStatus rs = redistribute_host(t);
        if (rs != pmSuccess) return rs;
    }
    for (size_t i = 0; i < ns; ++i) {
        AddressSpace* a = t->spaces[i];
        std::lock_guard<std::mutex> g(a->mu);
        for (Subtask& s : t->subtasks)
            for (const Record& r : s.mem[i].writes) {
                for (size_t q = 0; q < std::max<size_t>(r.count, 1); ++q)
                    a->dev_valid.remove(r.offset + q * r.step, r.offset + q * r.step + r.size);
            }
    }
    if (err.load() == pmStatusUnavailable) return fail(pmStatusUnavailable, "task timed out");
    if (err.load() != pmSuccess) return fail(static_cast<pmStatus>(err.load()), "CPU subtask callback failed");
    return pmSuccess;
}

static void finish_task(Task* t, pmStatus st, const std::string& msg) {
    Controller& c = ctl();
    for (Subtask& s : t->subtasks) {  // a failed task's private copies (its work has drained)
        for (char* p : s.dev_shadow)
            if (p) pmb_free_async(p, c.copy_stream);
        s.dev_shadow.clear();
        s.host_shadow.clear();
    }
    c.dev_held -= static_cast<int64_t>(t->reserved_held);
    t->reserved_held = 0;
    for (AddressSpace* a : t->spaces) {
        bool free_now = false;
        {
            std::lock_guard<std::mutex> g(c.mu);
            a->users--;
            free_now = a->released && a->users == 0;
            if (free_now) c.spaces.erase(a);
        }
        if (free_now) free_space(a);
    }
    if (st == pmSuccess && t->callbacks->cb.taskCompletionCallback) st = t->callbacks->cb.taskCompletionCallback(t->info);
    {
        std::lock_guard<std::mutex> g(t->mu);
        if (t->status == pmSuccess) t->status = st;
        if (!msg.empty() && t->error.empty()) t->error = msg;
        t->t_end = now_s();
        t->state = 2;
    }
    t->cv.notify_all();
}

static void stub_main() {
    Controller& c = ctl();
    if (c.has_gpu) pmb_set_device(c.device);
    for (;;) {
        Task* t = nullptr;
        {
            std::unique_lock<std::mutex> lk(c.qmu);
            c.qcv.wait(lk, [&] { return c.stopping || !c.queue.empty(); });
            if (c.queue.empty()) return;
            t = c.queue.front();
            c.queue.pop_front();
        }
        t->t_start = now_s();
        t->state = 1;
        if (t->deadline > 0 && now_s() > t->deadline) {
            finish_task(t, pmStatusUnavailable, "task timed out before it started");
            continue;
        }
        pmStatus st = run_dd(t, t->on_gpu ? c.gpu_info : c.cpu_info);
        if (st == pmSuccess) st = plan_reduction(t);
        if (st == pmSuccess) {
            if (t->on_gpu) {
                // Admission: a free slot, then device memory.  While tasks are in
                // flight their completion frees both, so wait for one and retry;
                // with nothing in flight a task that still does not fit fails.
                const double ta = now_s();
                {
                    std::unique_lock<std::mutex> lk(c.qmu);
                    c.icv.wait(lk, [&] { return c.inflight.size() < c.max_inflight; });
                }
                c.stats.slot_ns += ns_since(ta);
                const double tm = now_s();
                size_t need = 0;
                for (;;) {
                    if (admit(t, &need)) break;
                    std::unique_lock<std::mutex> lk(c.qmu);
                    if (c.inflight.empty()) break;
                    const size_t before = c.inflight.size();
                    c.icv.wait_for(lk, std::chrono::milliseconds(50), [&] { return c.inflight.size() < before; });
                }
                const bool fits = admit(t, &need);
                c.stats.mem_ns += ns_since(tm);
                c.stats.admit_ns += ns_since(ta);
                const double tl = now_s();
                st = fits ? stage_and_launch_gpu(t)
                          : fail(pmMemoryError, "task needs %zu bytes of device memory; not available", need);
                c.stats.stub_ns += ns_since(tl);
                if (st == pmSuccess) {
                    std::lock_guard<std::mutex> lk(c.qmu);
                    c.inflight.push_back(t);
                    c.icv.notify_all();
                    continue;
                }
                // Work already enqueued must drain before the task is reported.
                pmb_device_synchronize();
            } else {
                st = run_cpu_task(t);
            }
        }
        finish_task(t, st, st == pmSuccess ? "" : t_last_error);
    }
}

static void completer_main() {
    Controller& c = ctl();
    if (c.has_gpu) pmb_set_device(c.device);
    // Tasks finish in the order the device completes them, not the order they
    // were issued: a small task is not held behind a large one.
    std::vector<Task*> polled;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(c.qmu);
            c.icv.wait(lk, [&] { return c.stopping || !c.inflight.empty(); });
            if (c.inflight.empty()) return;
            polled.assign(c.inflight.begin(), c.inflight.end());
        }
        bool any = false;
        for (Task* t : polled) {
            const int st = pmb_event_query(t->done_event);
            if (st == PMB_STATUS_UNAVAILABLE) continue;
            any = true;
            {
                std::lock_guard<std::mutex> lk(c.qmu);
                c.inflight.erase(std::find(c.inflight.begin(), c.inflight.end(), t));
            }
            c.icv.notify_all();
            finish_task(t, st == PMB_SUCCESS ? pmSuccess : pmGraphicsCardError,
                        st == PMB_SUCCESS ? "" : std::string(pmb_last_error()));
        }
        if (!any) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

static pmStatus ensure_init() {
    return ctl().initialized ? pmSuccess : fail(pmInitializationFailure, "pmInitialize has not been called");
}

}  // namespace pmr

// ===========================================================================
// public API
// ===========================================================================
namespace pm {

using namespace pmr;

const char* pmGetLibVersion() { return "pmlib-b200 1_0_0"; }

const char* pmGetLastError() { return t_last_error.c_str(); }

pmStatus pmInitialize() {
    Controller& c = ctl();
    std::lock_guard<std::mutex> g(c.mu);
    if (c.initialized) return pmSuccess;
    int n = 0;
    pmb_device_count(&n);
    const char* dv = getenv("PMB_DEVICE");
    c.device = dv ? atoi(dv) : 0;
    c.has_gpu = n > c.device && pmb_device_supported(c.device);
    std::memset(c.cpu_info.name, 0, sizeof(c.cpu_info.name));
    std::snprintf(c.cpu_info.name, MAX_NAME_STR_LEN, "host CPU");
    std::snprintf(c.cpu_info.description, MAX_DESC_STR_LEN, "%u hardware threads", std::thread::hardware_concurrency());
    c.cpu_info.deviceHandle = &c.cpu_info;
    c.cpu_info.deviceType = CPU;
    c.cpu_info.host = 0;
    c.cpu_info.deviceIdOnHost = 0;
    c.cpu_info.deviceIdInCluster = 0;
    if (c.has_gpu) {
        if (pmb_set_device(c.device) != PMB_SUCCESS) return dev_fail(PMB_GRAPHICS_CARD_ERROR, "device selection");
        int sms = 0, ma = 0, mi = 0;
        pmb_device_properties(c.device, c.gpu_info.name, MAX_NAME_STR_LEN, &sms, &ma, &mi);
        std::snprintf(c.gpu_info.description, MAX_DESC_STR_LEN, "sm_%d%d, %d SMs", ma, mi, sms);
        c.gpu_info.deviceHandle = &c.gpu_info;
        c.gpu_info.deviceType = GPU_CUDA;
        c.gpu_info.host = 0;
        c.gpu_info.deviceIdOnHost = static_cast<uint>(c.device);
        c.gpu_info.deviceIdInCluster = 1;
        PMR_DEV(pmb_stream_create(&c.copy_stream));
        PMR_DEV(pmb_stream_create(&c.fetch_stream));
        const char* ns = getenv("PMB_STREAMS");
        c.streams.resize(ns && atoi(ns) > 0 ? static_cast<size_t>(atoi(ns)) : 16);
        for (auto& s : c.streams) PMR_DEV(pmb_stream_create(&s));
        PMR_DEV(pmb_mempool_retain(c.device));
        PMR_DEV(pmb_malloc(&c.dev_device_info, sizeof(pmDeviceInfo)));
        PMR_DEV(pmb_memcpy_async(c.dev_device_info, &c.gpu_info, sizeof(pmDeviceInfo), PMB_H2D, c.copy_stream));
        PMR_DEV(pmb_malloc(&c.dev_status, sizeof(pmStatus)));
        PMR_DEV(pmb_stream_synchronize(c.copy_stream));
        const char* rv = getenv("PMLIB_CUDA_MEM_PER_CARD_RESERVED_FOR_EXTERNAL_USE");
        c.reserve_bytes = rv ? static_cast<size_t>(atoll(rv)) : (size_t(512) << 20);
        size_t fr = 0, tot = 0;
        PMR_DEV(pmb_mem_get_info(&fr, &tot));
        c.dev_budget = fr > c.reserve_bytes ? static_cast<int64_t>((fr - c.reserve_bytes) / 10 * 9) : 0;
        c.dev_held = 0;
        // Map the budget into the stream-ordered pool now: growing the pool
        // while tasks run stalls their kernels and copies.
        const char* pr = getenv("PMB_POOL_RESERVE_BYTES");
        const size_t pool_want = std::min(pr ? static_cast<size_t>(atoll(pr)) : static_cast<size_t>(c.dev_budget),
                                          static_cast<size_t>(c.dev_budget));
        if (pool_want) PMR_DEV(pmb_mempool_reserve(c.device, pool_want, nullptr));
        const char* pv = getenv("PMB_PINNED_CACHE_BYTES");
        c.pin_limit = pv ? static_cast<size_t>(atoll(pv)) : (size_t(16) << 30);
        c.eager_writeback = env_flag("PMB_EAGER_WRITEBACK");
        const char* bg = getenv("PMB_BATCH_GROUPS");
        c.batch_groups = bg && atoi(bg) > 0 ? static_cast<size_t>(atoi(bg)) : 16;
        c.batch_off = env_flag("PMB_NO_BATCH");
        const char* mv = getenv("PMB_MAX_INFLIGHT");
        c.max_inflight = mv && atoi(mv) > 0 ? static_cast<size_t>(atoi(mv)) : 64;
    }
    c.stopping = false;
    c.stub = std::thread(stub_main);
    c.completer = std::thread(completer_main);
    c.initialized = true;
    return pmSuccess;
}

pmStatus pmFinalize() {
    Controller& c = ctl();
    if (!c.initialized) return pmSuccess;
    {
        std::lock_guard<std::mutex> lk(c.qmu);
        c.stopping = true;
    }
    c.qcv.notify_all();
    c.icv.notify_all();
    if (c.stub.joinable()) c.stub.join();
    if (c.completer.joinable()) c.completer.join();
    std::lock_guard<std::mutex> g(c.mu);
    if (c.has_gpu) pmb_device_synchronize();
    // Address spaces first: freeing a device mirror is ordered on the fetch stream.
    for (AddressSpace* a : c.spaces) free_space(a);
    c.spaces.clear();
    if (c.has_gpu) {
        pmb_stream_synchronize(c.fetch_stream);
        for (void* s : c.streams) pmb_stream_destroy(s);
        c.streams.clear();
        pmb_stream_destroy(c.copy_stream);
        pmb_stream_destroy(c.fetch_stream);
        pmb_free(c.dev_device_info);
        pmb_free(c.dev_status);
    }
    for (auto& kv : c.pin_free) pmb_host_free(kv.second);
    c.pin_free.clear();
    c.pin_cached = 0;
    for (auto& kv : c.files) munmap(kv.second.first, kv.second.second);
    c.files.clear();
    c.callbacks.clear();
    c.initialized = false;
    return pmSuccess;
}

uint pmGetHostId() { return 0; }
uint pmGetHostCount() { return 1; }

pmStatus pmRegisterCallbacks(const char* pKey, pmCallbacks pCallbacks, pmCallbackHandle* pCallbackHandle) {
    if (ensure_init() != pmSuccess) return pmInitializationFailure;
    if (!pKey || !pCallbackHandle) return fail(pmInvalidKey, "null key or handle");
    if (strlen(pKey) >= MAX_CB_KEY_LEN) return fail(pmMaxKeyLengthExceeded, "callback key longer than %zu", MAX_CB_KEY_LEN - 1);
    if (pCallbacks.subtask_gpu_cuda && pCallbacks.subtask_gpu_custom)
        return fail(pmInvalidCallbacks, "subtask_gpu_cuda and subtask_gpu_custom are both set");
    Controller& c = ctl();
    std::lock_guard<std::mutex> g(c.mu);
    for (auto& cs : c.callbacks)
        if (cs->key == pKey) return fail(pmInvalidKey, "callback key '%s' already registered", pKey);
    c.callbacks.emplace_back(new CallbackSet{pKey, pCallbacks});
    *pCallbackHandle = c.callbacks.back().get();
    return pmSuccess;
}

pmStatus pmReleaseCallbacks(pmCallbackHandle pCallbackHandle) {
    Controller& c = ctl();
    std::lock_guard<std::mutex> g(c.mu);
    for (auto it = c.callbacks.begin(); it != c.callbacks.end(); ++it)
        if (it->get() == pCallbackHandle) {
            c.callbacks.erase(it);
            return pmSuccess;
        }
    return fail(pmInvalidKey, "unknown callback handle");
}

pmStatus pmCreateMemory(size_t pLength, pmMemHandle* pMemHandle) {
    if (ensure_init() != pmSuccess) return pmInitializationFailure;
    if (!pMemHandle) return fail(pmInvalidIndex, "null handle");
    Controller& c = ctl();
    std::unique_ptr<AddressSpace> a(new AddressSpace);
    a->length = pLength;  // host and device copies are allocated on first use
    std::lock_guard<std::mutex> g(c.mu);
    c.spaces.insert(a.get());
    *pMemHandle = a.release();
    return pmSuccess;
}

pmStatus pmCreateMemory2D(size_t pRows, size_t pCols, pmMemHandle* pMemHandle) {
    const pmStatus st = pmCreateMemory(pRows * pCols, pMemHandle);
    if (st == pmSuccess) {
        AddressSpace* a = static_cast<AddressSpace*>(*pMemHandle);
        a->rows = pRows;
        a->cols = pCols;
    }
    return st;
}

pmStatus pmReleaseMemory(pmMemHandle pMemHandle) {
    Controller& c = ctl();
    AddressSpace* a = space_of(pMemHandle);
    if (!a) return fail(pmUnrecognizedMemory, "unknown memory handle");
    bool free_now;
    {
        std::lock_guard<std::mutex> g(c.mu);
        a->released = true;
        free_now = a->users == 0;
        if (free_now) c.spaces.erase(a);
    }
    if (free_now) {
        if (a->last_access) pmb_event_synchronize(a->last_access);
        free_space(a);
    }
    return pmSuccess;
}

pmStatus pmFetchMemory(pmMemHandle pMemHandle) {
    AddressSpace* a = space_of(pMemHandle);
    if (!a) return fail(pmUnrecognizedMemory, "unknown memory handle");
    if (ctl().has_gpu) pmb_set_device(ctl().device);
    std::lock_guard<std::mutex> g(a->mu);
    return fetch_range(a, 0, a->length);
}

pmStatus pmFetchMemoryRange(pmMemHandle pMemHandle, size_t pOffset, size_t pLength) {
    AddressSpace* a = space_of(pMemHandle);
    if (!a) return fail(pmUnrecognizedMemory, "unknown memory handle");
    if (pOffset + pLength > a->length) return fail(pmInvalidOffset, "range beyond the address space");
    if (ctl().has_gpu) pmb_set_device(ctl().device);
    std::lock_guard<std::mutex> g(a->mu);
    return fetch_range(a, pOffset, pOffset + pLength);
}

pmStatus pmGetRawMemPtr(pmMemHandle pMemHandle, pmRawMemPtr* pPtr) {
    AddressSpace* a = space_of(pMemHandle);
    if (!a || !pPtr) return fail(pmUnrecognizedMemory, "unknown memory handle");
    std::lock_guard<std::mutex> g(a->mu);
    const pmStatus hs = ensure_host(a);
    if (hs != pmSuccess) return hs;
    // The caller may now write the host copy: device bytes that are not newer
    // than the host are no longer trusted (they are re-staged on next use).
    RangeSet keep;
    for (auto& kv : a->host_stale.map()) keep.add(kv.first, kv.second);
    a->dev_valid = keep;
    *pPtr = a->host;
    return pmSuccess;
}

static pmStatus subscribe(pmTaskHandle pTaskHandle, ulong pSubtaskId, uint pMemIndex, pmSubscriptionType pType,
                          const Record& r) {
    Task* t = static_cast<Task*>(pTaskHandle);
    if (!t || t_dd.task != t) return fail(pmInvalidCommand, "pmSubscribeToMemory outside a data-distribution callback");
    if (pSubtaskId >= t->subtasks.size()) return fail(pmInvalidIndex, "subtask %lu out of range", pSubtaskId);
    if (pMemIndex >= t->spaces.size()) return fail(pmInvalidIndex, "memory index %u out of range", pMemIndex);
    AddressSpace* a = t->spaces[pMemIndex];
    if (r.count && r.size && (r.hi() > a->length || (r.count > 1 && r.step < r.size)))
        return fail(pmInvalidOffset, "subscription [%zu, %zu) outside the %zu-byte address space or overlapping",
                    r.lo(), r.hi(), a->length);
    const pmMemType mt = t->mem[pMemIndex].memType;
    if (pType != READ_SUBSCRIPTION && (mt == READ_ONLY || mt == READ_ONLY_LAZY))
        return fail(pmInvalidCommand, "write subscription on a read-only address space");
    if (pType != WRITE_SUBSCRIPTION && (mt == WRITE_ONLY || mt == WRITE_ONLY_LAZY))
        return fail(pmInvalidCommand, "read subscription on a write-only address space");
    SubtaskMem& m = t->subtasks[pSubtaskId].mem[pMemIndex];
    if (pType != WRITE_SUBSCRIPTION) m.reads.push_back(r);
    if (pType != READ_SUBSCRIPTION) m.writes.push_back(r);
    return pmSuccess;
}

pmStatus pmSubscribeToMemory(pmTaskHandle pTaskHandle, pmDeviceHandle, ulong pSubtaskId, pmSplitInfo&, uint pMemIndex,
                             pmSubscriptionType pSubscriptionType, const pmSubscriptionInfo& pSubscriptionInfo) {
    Record r;
    r.offset = pSubscriptionInfo.offset;
    r.size = pSubscriptionInfo.length;
    r.step = pSubscriptionInfo.length;
    r.count = pSubscriptionInfo.length ? 1 : 0;
    return subscribe(pTaskHandle, pSubtaskId, pMemIndex, pSubscriptionType, r);
}

pmStatus pmSubscribeToMemory(pmTaskHandle pTaskHandle, pmDeviceHandle, ulong pSubtaskId, pmSplitInfo&, uint pMemIndex,
                             pmSubscriptionType pSubscriptionType, const pmScatteredSubscriptionInfo& pInfo) {
    Record r;
    r.offset = pInfo.offset;
    r.size = pInfo.size;
    r.step = pInfo.step;
    r.count = pInfo.count;
    return subscribe(pTaskHandle, pSubtaskId, pMemIndex, pSubscriptionType, r);
}

// pmSubscriptionManager::RegisterRedistribution (pmSubscriptionManager.cpp:861-877):
// pOffset is relative to the start of the subtask's write range of the
// address space; zero-length ranges are ignored.
pmStatus pmRedistributeData(pmTaskHandle pTaskHandle, pmDeviceHandle, ulong pSubtaskId, pmSplitInfo&, uint pMemIndex,
                            size_t pOffset, size_t pLength, uint pOrder) {
    Task* t = task_of(pTaskHandle);
    if (!t) return fail(pmInvalidIndex, "unknown task handle");
    if (pMemIndex >= t->spaces.size() || pSubtaskId >= t->subtasks.size())
        return fail(pmInvalidIndex, "address space %u or subtask %lu out of range", pMemIndex, pSubtaskId);
    if (!pLength) return pmSuccess;
    size_t wlo, whi;
    consolidated(t->subtasks[pSubtaskId].mem[pMemIndex].writes, wlo, whi);
    if (whi <= wlo) return fail(pmInvalidIndex, "subtask %lu writes nothing of address space %u", pSubtaskId, pMemIndex);
    const size_t len = t->spaces[pMemIndex]->length;
    if (pOffset > len || pLength > len || wlo + pOffset > len - pLength)
        return fail(pmInvalidIndex, "redistributed range [%zu, +%zu) outside address space %u", wlo + pOffset, pLength,
                    pMemIndex);
    std::lock_guard<std::mutex> g(t->redist_mu);
    if (!t->redist_open) return fail(pmInvalidCommand, "pmRedistributeData outside a data-redistribution callback");
    RedistRecord r;
    r.order = pOrder;
    r.subtask = pSubtaskId;
    r.seq = t->redist[pMemIndex].size();
    r.offset = wlo + pOffset;
    r.length = pLength;
    t->redist[pMemIndex].push_back(r);
    return pmSuccess;
}

pmStatus pmSetCudaLaunchConf(pmTaskHandle pTaskHandle, pmDeviceHandle, ulong pSubtaskId, pmSplitInfo&,
                             pmCudaLaunchConf& pCudaLaunchConf) {
    Task* t = static_cast<Task*>(pTaskHandle);
    if (!t || t_dd.task != t) return fail(pmInvalidCommand, "pmSetCudaLaunchConf outside a data-distribution callback");
    if (pSubtaskId >= t->subtasks.size()) return fail(pmInvalidIndex, "subtask %lu out of range", pSubtaskId);
    t->subtasks[pSubtaskId].conf = pCudaLaunchConf;
    t->subtasks[pSubtaskId].has_conf = true;
    return pmSuccess;
}

pmStatus pmReserveCudaGlobalMem(pmTaskHandle pTaskHandle, pmDeviceHandle, ulong pSubtaskId, pmSplitInfo&, size_t pSize) {
    Task* t = static_cast<Task*>(pTaskHandle);
    if (!t || t_dd.task != t) return fail(pmInvalidCommand, "pmReserveCudaGlobalMem outside a data-distribution callback");
    if (pSubtaskId >= t->subtasks.size()) return fail(pmInvalidIndex, "subtask %lu out of range", pSubtaskId);
    t->subtasks[pSubtaskId].reserved = pSize;
    return pmSuccess;
}

pmStatus pmSubmitTask(pmTaskDetails pTaskDetails, pmTaskHandle* pTaskHandle) {
    if (ensure_init() != pmSuccess) return pmInitializationFailure;
    Controller& c = ctl();
    if (!pTaskHandle) return fail(pmInvalidIndex, "null task handle");
    if (pTaskDetails.taskMemCount > MAX_MEM_SECTIONS_PER_TASK)
        return fail(pmInvalidIndex, "%u address spaces (maximum %zu)", pTaskDetails.taskMemCount, MAX_MEM_SECTIONS_PER_TASK);
    if (pTaskDetails.taskMemCount && !pTaskDetails.taskMem) return fail(pmInvalidIndex, "null taskMem");
    std::unique_ptr<Task> t(new Task);
    {
        std::lock_guard<std::mutex> g(c.mu);
        for (auto& cs : c.callbacks)
            if (cs.get() == pTaskDetails.callbackHandle) t->callbacks = cs.get();
    }
    if (!t->callbacks) return fail(pmInvalidCallbacks, "unknown callback handle");
    const pmCallbacks& cb = t->callbacks->cb;
    t->details = pTaskDetails;
    if (pTaskDetails.taskConf && pTaskDetails.taskConfLength)
        t->conf.assign(static_cast<char*>(pTaskDetails.taskConf),
                       static_cast<char*>(pTaskDetails.taskConf) + pTaskDetails.taskConfLength);
    for (uint i = 0; i < pTaskDetails.taskMemCount; ++i) {
        AddressSpace* a = space_of(pTaskDetails.taskMem[i].memHandle);
        if (!a) return fail(pmUnrecognizedMemory, "taskMem[%u] is not a live address space", i);
        if (pTaskDetails.taskMem[i].memType >= MAX_MEM_TYPE) return fail(pmInvalidIndex, "taskMem[%u] has no memType", i);
        t->mem.push_back(pTaskDetails.taskMem[i]);
        t->spaces.push_back(a);
    }
    t->subtasks.resize(pTaskDetails.subtaskCount);
    for (ulong i = 0; i < pTaskDetails.subtaskCount; ++i) {
        t->subtasks[i].id = i;
        t->subtasks[i].mem.resize(t->spaces.size());
    }
    t->info.taskHandle = t.get();
    t->info.taskConf = t->conf.empty() ? nullptr : t->conf.data();
    t->info.taskConfLength = static_cast<uint>(t->conf.size());
    t->info.taskId = pTaskDetails.taskId;
    t->info.subtaskCount = pTaskDetails.subtaskCount;
    t->info.priority = pTaskDetails.priority;
    t->info.originatingHost = 0;
    const bool gpu_cb = cb.subtask_gpu_cuda || cb.subtask_gpu_custom;
    bool gpu_ok = gpu_cb && c.has_gpu;
    if (gpu_ok && cb.deviceSelection) gpu_ok = cb.deviceSelection(t->info, c.gpu_info);
    if (gpu_ok) {
        t->on_gpu = true;
        if (pmb_event_create(&t->done_event, 0) != PMB_SUCCESS) return dev_fail(PMB_GRAPHICS_CARD_ERROR, "event");
    } else if (cb.subtask_cpu && (!cb.deviceSelection || cb.deviceSelection(t->info, c.cpu_info))) {
        t->on_gpu = false;
    } else if (!gpu_cb && !cb.subtask_cpu) {
        t->on_gpu = false;  // placement-only task: data distribution runs, nothing executes
    } else {
        return fail(pmNoCompatibleDevice, gpu_cb ? "no supported CUDA device for this task" : "task has no usable subtask callback");
    }
    t->t_submit = now_s();
    if (pTaskDetails.timeOutInSecs > 0 && pTaskDetails.timeOutInSecs < INT32_MAX)
        t->deadline = t->t_submit + pTaskDetails.timeOutInSecs;
    Task* raw = t.release();
    {
        std::lock_guard<std::mutex> g(c.mu);
        c.tasks.insert(raw);
        for (AddressSpace* a : raw->spaces) a->users++;
    }
    {
        std::lock_guard<std::mutex> lk(c.qmu);
        c.queue.push_back(raw);
    }
    c.qcv.notify_all();
    *pTaskHandle = raw;
    return pmSuccess;
}

pmStatus pmWaitForTaskCompletion(pmTaskHandle pTaskHandle) {
    Task* t = task_of(pTaskHandle);
    if (!t) return fail(pmInvalidIndex, "unknown task handle");
    std::unique_lock<std::mutex> lk(t->mu);
    if (t->deadline > 0) {
        const auto dl = std::chrono::steady_clock::time_point(std::chrono::duration_cast<std::chrono::steady_clock::duration>(
            std::chrono::duration<double>(t->deadline)));
        if (!t->cv.wait_until(lk, dl, [&] { return t->state.load() == 2; }))
            return fail(pmStatusUnavailable, "task timed out after %d s", t->details.timeOutInSecs);
    } else {
        t->cv.wait(lk, [&] { return t->state.load() == 2; });
    }
    if (t->status != pmSuccess) t_last_error = t->error;
    return t->status;
}

pmStatus pmGetTaskExecutionTimeInSecs(pmTaskHandle pTaskHandle, double* pTime) {
    const pmStatus st = pmWaitForTaskCompletion(pTaskHandle);
    Task* t = task_of(pTaskHandle);
    if (!t || !pTime) return fail(pmInvalidIndex, "unknown task handle");
    *pTime = t->t_end - t->t_start;
    return st;
}

pmStatus pmReleaseTask(pmTaskHandle pTaskHandle) {
    Task* t = task_of(pTaskHandle);
    if (!t) return fail(pmInvalidIndex, "unknown task handle");
    {
        std::unique_lock<std::mutex> lk(t->mu);
        t->cv.wait(lk, [&] { return t->state.load() == 2; });  // even after a timeout: resources are in use
    }
    const pmStatus st = t->status;
    {
        std::lock_guard<std::mutex> g(ctl().mu);
        ctl().tasks.erase(t);
    }
    if (t->done_event) pmb_event_destroy(t->done_event);
    delete t;
    return st;
}

pmStatus pmReleaseTaskAndResources(pmTaskDetails pTaskDetails, pmTaskHandle pTaskHandle) {
    const pmStatus st = pmReleaseTask(pTaskHandle);
    pmReleaseCallbacks(pTaskDetails.callbackHandle);
    for (uint i = 0; i < pTaskDetails.taskMemCount; ++i) pmReleaseMemory(pTaskDetails.taskMem[i].memHandle);
    return st;
}

void* pmGetScratchBufferHostFunc(pmTaskHandle pTaskHandle, pmDeviceHandle, ulong pSubtaskId, pmSplitInfo&,
                                 pmScratchBufferType pScratchBufferType, size_t pBufferSize) {
    Task* t = static_cast<Task*>(pTaskHandle);
    if (!t || pSubtaskId >= t->subtasks.size()) return nullptr;
    auto& m = t->subtasks[pSubtaskId].scratch;
    auto it = m.find(pScratchBufferType);
    if (it == m.end()) {
        if (!pBufferSize) return nullptr;
        it = m.emplace(pScratchBufferType, std::vector<char>(pBufferSize, 0)).first;
    }
    return it->second.data();
}

pmStatus pmReleaseScratchBuffer(pmTaskHandle pTaskHandle, pmDeviceHandle, ulong pSubtaskId, pmSplitInfo&,
                                pmScratchBufferType pScratchBufferType) {
    Task* t = static_cast<Task*>(pTaskHandle);
    if (!t || pSubtaskId >= t->subtasks.size()) return fail(pmInvalidIndex, "unknown subtask");
    t->subtasks[pSubtaskId].scratch.erase(pScratchBufferType);
    return pmSuccess;
}

// pmTask::GetLastReductionScratchBuffer (pmTask.cpp:862-865): NULL when the
// task reduced nothing or its subtasks made no REDUCTION_TO_REDUCTION buffer.
void* pmGetLastReductionScratchBuffer(pmTaskHandle pTaskHandle) {
    Task* t = task_of(pTaskHandle);
    return t ? t->last_reduction_scratch : nullptr;
}

// pmRedistributor::GetRedistributionMetadata (pmRedistributor.cpp:296-322):
// (order, bytes) per order, ascending; valid until the task is released.
pmRedistributionMetadata* pmGetRedistributionMetadata(pmTaskHandle pTaskHandle, uint pMemIndex, ulong* pCount) {
    if (pCount) *pCount = 0;
    Task* t = task_of(pTaskHandle);
    if (!t || pMemIndex >= t->redist_meta.size() || t->redist_meta[pMemIndex].empty()) return nullptr;
    if (pCount) *pCount = t->redist_meta[pMemIndex].size();
    return t->redist_meta[pMemIndex].data();
}

// pmPublicDefinitions.cpp:779-815: the built-in callback of an (operation,
// data type) pair, NULL for values outside the enums.
pmDataReductionCallback pmGetSubtaskReductionCallbackImpl(pmReductionOpType pOperation, pmReductionDataType pDataType) {
    if (pOperation < 0 || pOperation >= MAX_REDUCTION_OP_TYPES || pDataType < 0 || pDataType >= MAX_REDUCTION_DATA_TYPES)
        return nullptr;
    return kBuiltinReduction[pOperation][pDataType];
}

// Folds subtask 2's private copies into subtask 1's (host copies; called from
// reduction callbacks), over every reducible address space both wrote
// (pmReducer::ReduceSubtasks, pmReducer.cpp:1073-1296).
pmStatus pmReduceSubtasks(pmTaskHandle pTaskHandle, pmDeviceHandle, unsigned long pSubtask1Id, pmSplitInfo&,
                          pmDeviceHandle, unsigned long pSubtask2Id, pmSplitInfo&, pmReductionOpType pOperation,
                          pmReductionDataType pDataType) {
    Task* t = task_of(pTaskHandle);
    if (!t) return fail(pmInvalidIndex, "unknown task handle");
    if (pSubtask1Id >= t->subtasks.size() || pSubtask2Id >= t->subtasks.size())
        return fail(pmInvalidIndex, "subtask %lu or %lu out of range", pSubtask1Id, pSubtask2Id);
    Subtask& s1 = t->subtasks[pSubtask1Id];
    Subtask& s2 = t->subtasks[pSubtask2Id];
    for (const ReduceSpace& rs : t->reduce) {
        const size_t i = rs.index;
        if (s1.host_shadow.size() <= i || s2.host_shadow.size() <= i || s1.host_shadow[i].empty() ||
            s2.host_shadow[i].empty())
            return fail(pmInvalidIndex, "subtasks %lu and %lu have no reduction copies of address space %zu",
                        pSubtask1Id, pSubtask2Id, i);
        if (s1.host_shadow[i].size() != s2.host_shadow[i].size())
            return fail(pmInvalidIndex, "reduction copies of address space %zu differ in length", i);
        const pmStatus st = host_reduce(pOperation, pDataType, s1.host_shadow[i].data(), s2.host_shadow[i].data(),
                                        s1.host_shadow[i].size());
        if (st != pmSuccess) return st;
    }
    return pmSuccess;
}

void* pmGetMappedFile(const char* pPath) {
    if (!pPath) return nullptr;
    std::lock_guard<std::mutex> g(ctl().mu);
    auto it = ctl().files.find(pPath);
    return it == ctl().files.end() ? nullptr : it->second.first;
}

pmStatus pmMapFile(const char* pPath) {
    if (!pPath || strlen(pPath) >= MAX_FILE_SIZE_LEN) return fail(pmInvalidKey, "bad path");
    const int fd = open(pPath, O_RDONLY);
    if (fd < 0) return fail(pmConfFileNotFound, "cannot open %s", pPath);
    struct stat sb;
    if (fstat(fd, &sb) != 0) {
        close(fd);
        return fail(pmConfFileNotFound, "cannot stat %s", pPath);
    }
    void* p = mmap(nullptr, sb.st_size ? sb.st_size : 1, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (p == MAP_FAILED) return fail(pmMemoryError, "mmap of %s failed", pPath);
    std::lock_guard<std::mutex> g(ctl().mu);
    ctl().files[pPath] = {p, static_cast<size_t>(sb.st_size ? sb.st_size : 1)};
    return pmSuccess;
}

pmStatus pmUnmapFile(const char* pPath) {
    std::lock_guard<std::mutex> g(ctl().mu);
    auto it = pPath ? ctl().files.find(pPath) : ctl().files.end();
    if (it == ctl().files.end()) return fail(pmInvalidKey, "file not mapped");
    munmap(it->second.first, it->second.second);
    ctl().files.erase(it);
    return pmSuccess;
}

pmStatus pmMapFiles(const char* const* pPaths, uint pFileCount) {
    for (uint i = 0; i < pFileCount; ++i) {
        const pmStatus st = pmMapFile(pPaths[i]);
        if (st != pmSuccess) return st;
    }
    return pmSuccess;
}

pmStatus pmUnmapFiles(const char* const* pPaths, uint pFileCount) {
    for (uint i = 0; i < pFileCount; ++i) {
        const pmStatus st = pmUnmapFile(pPaths[i]);
        if (st != pmSuccess) return st;
    }
    return pmSuccess;
}

}  // namespace pm

extern "C" int pmb_runtime_register_batch_groups(void* subtask_gpu_custom, void* batch_fn, int groups) {
    if (!subtask_gpu_custom || !batch_fn || groups < 0) return pm::pmInvalidIndex;
    pmr::register_batch(reinterpret_cast<pm::pmSubtaskCallback_GPU_Custom>(subtask_gpu_custom),
                        reinterpret_cast<pmr::BatchFn>(batch_fn), static_cast<size_t>(groups));
    return pm::pmSuccess;
}

extern "C" int pmb_runtime_register_batch(void* subtask_gpu_custom, void* batch_fn) {
    if (!subtask_gpu_custom || !batch_fn) return pm::pmInvalidIndex;
    pmr::register_batch(reinterpret_cast<pm::pmSubtaskCallback_GPU_Custom>(subtask_gpu_custom),
                        reinterpret_cast<pmr::BatchFn>(batch_fn), 0);
    return pm::pmSuccess;
}

extern "C" void pmb_runtime_stats(unsigned long long* h2d, unsigned long long* d2h, unsigned long long* gpu_subtasks,
                                  unsigned long long* batched) {
    pmr::Controller& c = pmr::ctl();
    if (h2d) *h2d = c.stats.h2d;
    if (d2h) *d2h = c.stats.d2h;
    if (gpu_subtasks) *gpu_subtasks = c.stats.gpu_subtasks;
    if (batched) *batched = c.stats.batched;
}

extern "C" void pmb_runtime_set_eager_writeback(int on) { pmr::ctl().eager_writeback = on != 0; }

extern "C" void pmb_runtime_timers(double* stub_s, double* admit_wait_s, double* pinned_alloc_s,
                                   unsigned long long* pinned_alloc_bytes) {
    pmr::Controller& c = pmr::ctl();
    if (stub_s) *stub_s = c.stats.stub_ns * 1e-9;
    if (admit_wait_s) *admit_wait_s = c.stats.admit_ns * 1e-9;
    if (pinned_alloc_s) *pinned_alloc_s = c.stats.pin_ns * 1e-9;
    if (pinned_alloc_bytes) *pinned_alloc_bytes = c.stats.pin_bytes;
}

extern "C" void pmb_runtime_admission(double* slot_wait_s, double* memory_wait_s, unsigned long long* evictions,
                                      unsigned long long* evicted_bytes) {
    pmr::Controller& c = pmr::ctl();
    if (slot_wait_s) *slot_wait_s = c.stats.slot_ns * 1e-9;
    if (memory_wait_s) *memory_wait_s = c.stats.mem_ns * 1e-9;
    if (evictions) *evictions = c.stats.evictions;
    if (evicted_bytes) *evicted_bytes = c.stats.evicted_bytes;
}

extern "C" void pmb_runtime_sentinel_stats(unsigned long long* copies, unsigned long long* bytes) {
    if (copies) *copies = pmr::ctl().stats.sentinel_copies;
    if (bytes) *bytes = pmr::ctl().stats.sentinel_bytes;
}

extern "C" double pmb_runtime_callback_seconds(void) { return pmr::ctl().stats.callback_ns * 1e-9; }

extern "C" void pmb_runtime_fetch_timers(double* host_s, double* wait_s, double* copy_s, unsigned long long* fetches) {
    pmr::Controller& c = pmr::ctl();
    if (host_s) *host_s = c.stats.fetch_host_ns * 1e-9;
    if (wait_s) *wait_s = c.stats.fetch_wait_ns * 1e-9;
    if (copy_s) *copy_s = c.stats.fetch_copy_ns * 1e-9;
    if (fetches) *fetches = c.stats.fetches;
}

extern "C" void pmb_runtime_reset_stats(void) {
    pmr::Controller& c = pmr::ctl();
    c.stats.slot_ns = 0;
    c.stats.callback_ns = 0;
    c.stats.fetch_host_ns = 0;
    c.stats.fetch_wait_ns = 0;
    c.stats.fetch_copy_ns = 0;
    c.stats.fetches = 0;
    c.stats.mem_ns = 0;
    c.stats.evictions = 0;
    c.stats.evicted_bytes = 0;
    c.stats.stub_ns = 0;
    c.stats.admit_ns = 0;
    c.stats.pin_ns = 0;
    c.stats.pin_bytes = 0;
    c.stats.h2d = 0;
    c.stats.d2h = 0;
    c.stats.gpu_subtasks = 0;
    c.stats.batched = 0;
}
