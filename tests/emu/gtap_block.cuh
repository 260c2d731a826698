// gtap_block.cuh -- TEST INFRASTRUCTURE: a CPU emulator of the block-mode task
// ABI (the entry points of include/gtap_block.cuh, after the reference's
// runtime/gtap_block.cuh).  One emulated block of GTAP_BLOCK_SIZE host threads
// runs every task, one task at a time, in the order GTAP_EMU_ORDER chooses
// (lifo, fifo, random with GTAP_EMU_SEED); all its threads run the task body,
// __syncthreads is a barrier among them, and `__shared__` variables are shared
// by them.  Kernel launches must go through emu_launch (cuda_runtime.h here).
// It checks the protocol block-mode code must follow:
//   * every thread reaches each join and each finish (a barrier that waits
//     more than a few seconds stops the program with an error);
//   * a frame is filled before it is read (new and freed frames are
//     poisoned); a retained child is released once, after it finished; a
//     release takes effect when the execution ends, as in the GPU runtime.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <random>
#include <vector>

#ifndef GTAP_GRID_SIZE
#define GTAP_GRID_SIZE 1
#endif
#ifndef GTAP_BLOCK_SIZE
#define GTAP_BLOCK_SIZE 32
#endif
#ifndef GTAP_NUM_QUEUES
#define GTAP_NUM_QUEUES 1
#endif

struct TaskContext;
extern const size_t __gtap_auto_task_data_size;

#ifdef GTAP_DIRECT_DISPATCH
void __gtap_dispatch(unsigned long long fn, void* frame, int tid, TaskContext* ctx);
#endif

inline int load_L2(int* p) { return __atomic_load_n(p, __ATOMIC_SEQ_CST); }
inline unsigned load_L2(unsigned* p) { return __atomic_load_n(p, __ATOMIC_SEQ_CST); }
inline void store_L2(int* p, int v) { __atomic_store_n(p, v, __ATOMIC_SEQ_CST); }
inline unsigned get_lane_id() { return threadIdx.x & 31u; }

namespace gtap_emu_block {

constexpr size_t kFrameBytes = 256;
constexpr unsigned char kPoison = 0xA5;

struct Rec {
    void (*fn)(void*, int, TaskContext*) = nullptr;
    int state = 0, parent = -1, pending = 0, since_join = 0;
    bool live = false, suspended = false, finished = false, retained = false;
    alignas(16) unsigned char frame[kFrameBytes];
};

struct Emu {
    std::mutex mu;   // spawns and releases come from any thread of the block
    std::deque<Rec> recs;
    std::vector<int> free_ids, staged, released;
    std::deque<int> ready;
    std::mt19937_64 rng{1};
    int order = 0, error = 0;
    // barrier
    std::mutex bmu;
    std::condition_variable bcv;
    int arrived = 0;
    unsigned long long generation = 0;
    // values thread 0 hands to the block
    int current = -1;
    bool decision = false;
};
inline Emu& emu() {
    static Emu e;
    return e;
}

inline void fail(int code, const char* what, int tid) {
    Emu& E = emu();
    if (!E.error) {
        E.error = code;
        fprintf(stderr, "block emulator: %s (task %d)\n", what, tid);
    }
}

// all GTAP_BLOCK_SIZE threads meet; a thread that waits too long ends the program
inline void barrier() {
    Emu& E = emu();
    std::unique_lock<std::mutex> lk(E.bmu);
    const unsigned long long gen = E.generation;
    if (++E.arrived == GTAP_BLOCK_SIZE) {
        E.arrived = 0;
        E.generation++;
        E.bcv.notify_all();
        return;
    }
    if (!E.bcv.wait_for(lk, std::chrono::seconds(10), [&] { return E.generation != gen; })) {
        fprintf(stderr, "block emulator: a barrier waited 10 s -- not every thread reached it\n");
        fflush(stderr);
        std::_Exit(3);
    }
}
inline void sync_hook() { barrier(); }

inline int alloc_id() {
    Emu& E = emu();
    int id;
    if (!E.free_ids.empty()) {
        id = E.free_ids.back();
        E.free_ids.pop_back();
    } else {
        id = (int)E.recs.size();
        E.recs.emplace_back();
    }
    Rec& r = E.recs[id];
    r = Rec();
    r.live = true;
    memset(r.frame, kPoison, kFrameBytes);
    return id;
}

inline void free_id(int id) {
    Emu& E = emu();
    Rec& r = E.recs[id];
    r.live = false;
    memset(r.frame, kPoison, kFrameBytes);
    E.free_ids.push_back(id);
}

inline void reset() {
    Emu& E = emu();
    E.recs.clear();
    E.free_ids.clear();
    E.ready.clear();
    E.staged.clear();
    E.released.clear();
    E.error = 0;
    const char* o = getenv("GTAP_EMU_ORDER");
    E.order = (o && !strcmp(o, "fifo")) ? 1 : (o && !strcmp(o, "random")) ? 2 : 0;
    const char* s = getenv("GTAP_EMU_SEED");
    E.rng.seed(s ? strtoull(s, nullptr, 10) : 1);
    emu_block_threads() = GTAP_BLOCK_SIZE;
    emu_sync_hook() = &sync_hook;
    if (__gtap_auto_task_data_size > kFrameBytes) fail(99, "frame larger than the emulator's records", -1);
}

}  // namespace gtap_emu_block

// ---------------------------------------------------------------------------
// device ABI
// ---------------------------------------------------------------------------
inline int __gtap_get_task_state(int tid) { return gtap_emu_block::emu().recs[tid].state; }

inline void* __gtap_spawn_task(TaskContext*, int self_tid, int* child_count, void (*func)(void*, int, TaskContext*),
                               int child_queue_idx, int* out_tid, bool retain_parent_result) {
    using namespace gtap_emu_block;
    Emu& E = emu();
    std::lock_guard<std::mutex> lk(E.mu);
    if (child_queue_idx < 0 || child_queue_idx >= GTAP_NUM_QUEUES) fail(1, "queue index out of range", self_tid);
    const int id = alloc_id();
    Rec& c = E.recs[id];
    c.fn = func;
    c.parent = self_tid;
#ifdef GTAP_ASSUME_NO_TASKWAIT
    c.parent = -1;
    (void)retain_parent_result;
#else
    c.retained = retain_parent_result;
    E.recs[self_tid].pending++;
    E.recs[self_tid].since_join++;
#endif
    if (child_count) ++*child_count;
    E.staged.push_back(id);
    if (out_tid) *out_tid = id;
    return c.frame;
}

// block-wide: every thread calls it; all get the same answer
inline bool __gtap_set_state_for_join_block(int tid, TaskContext*, int next_state, int) {
    using namespace gtap_emu_block;
    Emu& E = emu();
    barrier();   // every spawn of this execution is in
    if (threadIdx.x == 0) {
        Rec& r = E.recs[tid];
        r.state = next_state;
        const bool wait = r.since_join > 0 && r.pending > 0;
        r.since_join = 0;
        r.suspended = wait;
        E.decision = wait;
    }
    barrier();
    const bool d = E.decision;
    barrier();   // every thread has read it before it changes
    return d;
}

inline bool __gtap_set_state_for_join(int tid, int, int next_state, int q) {
    return __gtap_set_state_for_join_block(tid, nullptr, next_state, q);
}

inline void __gtap_finish_task(int tid, TaskContext*) {
    using namespace gtap_emu_block;
    Emu& E = emu();
    barrier();
    if (threadIdx.x == 0) {
        Rec& r = E.recs[tid];
        r.finished = true;
        if (r.pending > 0)
            for (size_t i = 0; i < E.recs.size(); ++i)
                if (E.recs[i].live && E.recs[i].parent == tid) E.recs[i].parent = -1;
        const int p = r.parent;
        if (p >= 0) {
            Rec& pr = E.recs[p];
            if (--pr.pending == 0 && pr.suspended) E.ready.push_back(p);
        }
    }
    barrier();
}

inline void* __gtap_get_task_data(int tid) { return gtap_emu_block::emu().recs[tid].frame; }

template <typename TaskType>
inline TaskType* __gtap_get_task_data(int tid) {
    return reinterpret_cast<TaskType*>(__gtap_get_task_data(tid));
}

// takes effect when the execution ends (the GPU block runtime defers it too)
inline void __gtap_release_task_id(int tid) {
    using namespace gtap_emu_block;
    Emu& E = emu();
    std::lock_guard<std::mutex> lk(E.mu);
    Rec& r = E.recs[tid];
    if (!r.live || !r.retained || !r.finished) {
        fail(99, "release of a task that is not a finished retained child", tid);
        return;
    }
    E.released.push_back(tid);
}

inline void __gtap_push_initial_task(void (*func)(void*, int, TaskContext*), int initial_queue_idx) {
    using namespace gtap_emu_block;
    Emu& E = emu();
    if (initial_queue_idx < 0 || initial_queue_idx >= GTAP_NUM_QUEUES) fail(1, "queue index out of range", 0);
    const int id = alloc_id();
    if (id != 0) fail(99, "the initial task is not task 0", id);
    E.recs[id].fn = func;
    E.ready.push_back(id);
}

// every thread of the block calls it
inline void __gtap_execute_task_loop_device() {
    using namespace gtap_emu_block;
    Emu& E = emu();
    barrier();   // the initial task and its frame are written
    for (;;) {
        if (threadIdx.x == 0) {
            int t = -1;
            if (!E.ready.empty() && !E.error) {
                if (E.order == 0) {
                    t = E.ready.back();
                    E.ready.pop_back();
                } else if (E.order == 1) {
                    t = E.ready.front();
                    E.ready.pop_front();
                } else {
                    const size_t i = (size_t)(E.rng() % E.ready.size());
                    t = E.ready[i];
                    E.ready[i] = E.ready.back();
                    E.ready.pop_back();
                }
                E.recs[t].suspended = false;
            }
            E.current = t;
        }
        barrier();
        const int t = E.current;
        if (t < 0) break;
        Rec& r = E.recs[t];
#if defined(GTAP_DIRECT_DISPATCH)
        __gtap_dispatch((unsigned long long)(void*)r.fn, r.frame, t, nullptr);
#else
        r.fn(r.frame, t, nullptr);
#endif
        barrier();
        if (threadIdx.x == 0) {
            if (!r.finished && !r.suspended) fail(99, "an execution returned without finishing or suspending", t);
            for (int id : E.released) free_id(id);
            E.released.clear();
            if (r.finished && !r.retained) free_id(t);
            for (int c : E.staged) E.ready.push_back(c);
            E.staged.clear();
        }
        barrier();
    }
    barrier();
    if (threadIdx.x == 0)
        for (size_t i = 0; i < E.recs.size() && !E.error; ++i)
            if (E.recs[i].live && !E.recs[i].finished) fail(99, "a task never ran to its end", (int)i);
}

// ---------------------------------------------------------------------------
// host API
// ---------------------------------------------------------------------------
inline cudaError_t gtap_initialize() {
    gtap_emu_block::reset();
    return cudaSuccess;
}
inline cudaError_t gtap_reset() {
    gtap_emu_block::reset();
    return cudaSuccess;
}
inline cudaError_t gtap_synchronize() { return cudaSuccess; }
inline cudaError_t gtap_finalize() { return cudaSuccess; }
inline cudaError_t gtap_get_runtime_error_code(int* code) {
    *code = gtap_emu_block::emu().error;
    return cudaSuccess;
}
inline cudaError_t gtap_check_runtime_error() { return gtap_emu_block::emu().error ? 1 : cudaSuccess; }
