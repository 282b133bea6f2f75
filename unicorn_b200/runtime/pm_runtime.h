// Internal declarations of the pm:: runtime (libpmlib.so).  Not installed:
// apps include pmPublicDefinitions.h / pmPublicUtilities.h only.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pmPublicDefinitions.h"
#include "pmPublicUtilities.h"

namespace pmr {

using namespace pm;

// Sorted, disjoint, non-adjacent set of byte ranges [lo, hi).
class RangeSet {
public:
    void add(size_t lo, size_t hi);
    void remove(size_t lo, size_t hi);
    bool covers(size_t lo, size_t hi) const;
    // Parts of [lo, hi) not in the set, appended to `out`.
    void missing(size_t lo, size_t hi, std::vector<std::pair<size_t, size_t>>& out) const;
    // Parts of [lo, hi) in the set, appended to `out`.
    void present(size_t lo, size_t hi, std::vector<std::pair<size_t, size_t>>& out) const;
    bool empty() const { return m_.empty(); }
    void clear() { m_.clear(); }
    size_t bytes() const;
    const std::map<size_t, size_t>& map() const { return m_; }

private:
    std::map<size_t, size_t> m_;  // lo -> hi
};

// `count` pieces of `size` bytes, `step` apart, the first at `offset`.
struct Record {
    size_t offset = 0, size = 0, step = 0, count = 0;
    size_t lo() const { return offset; }
    size_t hi() const { return count ? offset + (count - 1) * step + size : offset; }
    bool contiguous() const { return count <= 1 || step == size; }
};

struct AddressSpace {
    size_t length = 0;
    size_t rows = 0, cols = 0;  // pmCreateMemory2D layout (informational)
    char* host = nullptr;       // pinned host copy, allocated on first host use
    size_t host_cap = 0;        // bytes of the host allocation (>= length when reused)
    char* dev = nullptr;        // device mirror, allocated on first GPU use
    RangeSet dev_valid;         // bytes whose device copy is current
    RangeSet host_stale;        // bytes the device has newer than the host
    void* last_write = nullptr; // event after the last device write (owned)
    void* last_access = nullptr;// event after the last device read or write (owned)
    int users = 0;              // tasks submitted and not yet finished
    bool released = false;
    uint64_t lru = 0;
    std::mutex mu;
};

struct SubtaskMem {
    std::vector<Record> reads, writes;
};

struct Subtask {
    ulong id = 0;
    std::vector<SubtaskMem> mem;  // per task address space
    bool has_conf = false;
    pmCudaLaunchConf conf;
    size_t reserved = 0;
    std::map<int, std::vector<char>> scratch;  // pmScratchBufferType -> host buffer
    void* dev_scratch = nullptr;
    void* dev_reserved = nullptr;
    std::vector<void*> dev_compact;  // per address space
    pmSubtaskInfo info;              // device view handed to the GPU callback
    pmStatus status = pmSuccess;
    // Private copies of the reducible address spaces (tasks with a
    // dataReduction callback), over the range every subtask subscribes:
    // device copies for GPU subtasks, host copies on the CPU and for
    // reduction callbacks that run on the host.  Per task address space.
    std::vector<char*> dev_shadow;
    std::vector<std::vector<char>> host_shadow;
};

// One writable address space of a task with a dataReduction callback: the
// byte range [lo, hi) every writing subtask subscribes (reads and writes),
// the written part [wlo, whi), and the writing subtasks in id order.
struct ReduceSpace {
    size_t index = 0;
    size_t lo = 0, hi = 0, wlo = 0, whi = 0;
    std::vector<size_t> subtasks;
};

// One pmRedistributeData call: `length` bytes at `offset` of the address
// space (the subtask's write range start + the offset it passed) go to order
// `order`; ties broken by subtask id, then call sequence.
struct RedistRecord {
    unsigned int order = 0;
    size_t subtask = 0, seq = 0;
    size_t offset = 0, length = 0;
};

struct CallbackSet {
    std::string key;
    pmCallbacks cb;
};

struct Task;

using BatchFn = pmStatus (*)(const pmTaskInfo* task, const pmDeviceInfo* device, const pmSubtaskInfo* subtasks,
                             unsigned long count, void* stream);

struct Task {
    pmTaskDetails details;
    std::vector<char> conf;      // host copy of taskConf
    void* dev_conf = nullptr;    // device copy (subtask_gpu_cuda kernels dereference it)
    std::vector<pmTaskMem> mem;
    std::vector<AddressSpace*> spaces;
    std::vector<pmSubscriptionVisibilityType> views;  // resolved per address space
    CallbackSet* callbacks = nullptr;
    std::vector<Subtask> subtasks;
    pmTaskInfo info;             // host task info (taskConf = host copy)
    pmTaskInfo dev_info;         // taskConf = device copy
    bool on_gpu = false;
    void* done_event = nullptr;
    double t_submit = 0, t_start = 0, t_end = 0;
    size_t reserved_held = 0;    // reserved subtask memory and reduction copies counted against the device budget
    std::vector<ReduceSpace> reduce;  // reducible address spaces (dataReduction tasks)
    int reduce_op = -1, reduce_type = -1;  // built-in REDUCE_* callback, else -1 (the app's own callback)
    void* last_reduction_scratch = nullptr;  // REDUCTION_TO_REDUCTION buffer of the subtask all others folded into
    // Ordered redistribution (dataRedistribution callback): records per
    // address space, and after the task the (order, bytes) metadata of each.
    std::mutex redist_mu;
    std::vector<std::vector<RedistRecord>> redist;
    std::vector<std::vector<pmRedistributionMetadata>> redist_meta;
    bool redist_open = false;  // inside the redistribution callbacks
    double deadline = 0;         // 0: none
    std::atomic<int> state{0};   // 0 queued, 1 running, 2 done
    pmStatus status = pmSuccess;
    std::string error;
    std::mutex mu;
    std::condition_variable cv;
};

// Registers a whole-task GPU implementation for a subtask_gpu_custom callback:
// when every subtask of a task uses that callback with NATURAL views, the
// CUDA stub calls `batch` once per group of consecutive subtasks instead of
// once per subtask -- `groups` groups per task (0: PMB_BATCH_GROUPS, 16 by
// default), each launched as soon as its own inputs are staged.
// PMB_NO_BATCH=1 turns every hook off (per-subtask callbacks).
void register_batch(pmSubtaskCallback_GPU_Custom callback, BatchFn batch, size_t groups);

}  // namespace pmr

extern "C" {
// C entries for apps libraries (see register_batch).
int pmb_runtime_register_batch(void* subtask_gpu_custom, void* batch_fn);
int pmb_runtime_register_batch_groups(void* subtask_gpu_custom, void* batch_fn, int groups);
// Runtime statistics: bytes moved host->device / device->host, GPU callback
// invocations, batched launches; for tests and benchmarks.
void pmb_runtime_stats(unsigned long long* h2d_bytes, unsigned long long* d2h_bytes,
                       unsigned long long* gpu_subtasks, unsigned long long* batched_launches);
// Write back the bytes a GPU task writes at the end of the task, on the task's
// own stream (1), or leave them on the device until pmFetchMemory (0, the
// default; PMB_EAGER_WRITEBACK=1 sets 1 at pmInitialize).  Tasks issued after
// the call follow the new setting.
void pmb_runtime_set_eager_writeback(int on);
// Seconds the CUDA stub spent issuing GPU tasks (staging and launching) and
// waiting to admit them, and the pinned host allocations it made (seconds,
// bytes); for benchmarks.
void pmb_runtime_timers(double* stub_s, double* admit_wait_s, double* pinned_alloc_s,
                        unsigned long long* pinned_alloc_bytes);
// Admission: seconds waiting for a slot and for device memory, and the idle
// mirrors evicted to make room (count, bytes).
void pmb_runtime_admission(double* slot_wait_s, double* memory_wait_s, unsigned long long* evictions,
                           unsigned long long* evicted_bytes);
// Seconds spent inside subtask_gpu_custom callbacks (the apps' own launches).
double pmb_runtime_callback_seconds(void);
// Write-back of device results to host memory (pmFetchMemory, eviction):
// seconds getting host buffers, waiting for the producing tasks, copying
// (issue to completion); and the number of write-backs.
void pmb_runtime_fetch_timers(double* host_s, double* wait_s, double* copy_s, unsigned long long* fetches);
void pmb_runtime_reset_stats(void);
}
