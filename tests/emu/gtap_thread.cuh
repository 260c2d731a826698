// gtap_thread.cuh -- TEST INFRASTRUCTURE: a sequential CPU emulator of the
// thread-mode task ABI (the entry points of include/gtap_thread.cuh, after the
// reference's runtime/gtap_thread.cuh), so that the state machines
// gtap_b200.lower emits can be run on the host and their results checked,
// without a GPU.  It is not the runtime: it runs one task at a time, in an
// order chosen by GTAP_EMU_ORDER (lifo, fifo, or random with GTAP_EMU_SEED),
// and checks the protocol the lowered code must follow:
//   * a frame is filled before it is read: new frames are poisoned (0xA5) and
//     a freed frame is poisoned again, so a stale or unwritten read shows up
//     in the results;
//   * a join is given the number of children spawned since the last one;
//   * an execution ends in __gtap_finish_task or in a join that suspends;
//   * a retained child is released once, after it finished.
// Children become runnable after the body that spawned them returns, and a
// suspended parent when its last child finished, as on the GPU.  With
// GTAP_FRAME_WORDS the first 32 frame bytes are handed to
// __gtap_dispatch_words, as the drop-in header does.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <deque>
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
#ifndef GTAP_MAX_CHILD_TASKS
#define GTAP_MAX_CHILD_TASKS 32
#endif

struct TaskContext;
extern const size_t __gtap_auto_task_data_size;

#ifdef GTAP_DIRECT_DISPATCH
void __gtap_dispatch(unsigned long long fn, void* frame, int tid, TaskContext* ctx);
#endif
#ifdef GTAP_FRAME_WORDS
void __gtap_dispatch_words(unsigned long long fn, void* frame, int tid, TaskContext* ctx, int4 w0, int4 w1);
#endif

// the device helpers the drop-in header gives task code (include/gtap_device_util.cuh)
inline int load_L2(int* p) { return *p; }
inline unsigned load_L2(unsigned* p) { return *p; }
inline uint16_t load_L2_u16t(uint16_t* p) { return *p; }
inline int load_L2_acquire(int* p) { return *p; }
inline void store_L2(int* p, int v) { *p = v; }
inline void store_L2(unsigned* p, unsigned v) { *p = v; }
inline void store_L2_release(int* p, int v) { *p = v; }
inline int atomicCAS_acquire(int* p, int expected, int desired) {
    const int old = *p;
    if (old == expected) *p = desired;
    return old;
}
inline unsigned get_lane_id() { return 0; }
inline unsigned get_warp_id_in_block() { return 0; }
inline unsigned get_warp_id_global() { return 0; }

namespace gtap_emu {

constexpr size_t kFrameBytes = 256;
constexpr unsigned char kPoison = 0xA5;

struct Rec {
    void (*fn)(void*, int, TaskContext*) = nullptr;
    int state = 0, parent = -1, pending = 0, since_join = 0;
    bool live = false, suspended = false, finished = false, retained = false;
    alignas(16) unsigned char frame[kFrameBytes];
};

struct Emu {
    std::deque<Rec> recs;   // records never move while a task holds a frame pointer
    std::vector<int> free_ids, staged;
    std::deque<int> ready;
    std::mt19937_64 rng{1};
    int order = 0;   // 0 lifo, 1 fifo, 2 random
    int error = 0;
    long long executions = 0;
};
inline Emu& emu() {
    static Emu e;
    return e;
}

inline void fail(int code, const char* what, int tid) {
    Emu& E = emu();
    if (!E.error) {
        E.error = code;
        fprintf(stderr, "emulator: %s (task %d)\n", what, tid);
    }
}

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
    E.error = 0;
    E.executions = 0;
    const char* o = getenv("GTAP_EMU_ORDER");
    E.order = (o && !strcmp(o, "fifo")) ? 1 : (o && !strcmp(o, "random")) ? 2 : 0;
    const char* s = getenv("GTAP_EMU_SEED");
    E.rng.seed(s ? strtoull(s, nullptr, 10) : 1);
    if (__gtap_auto_task_data_size > kFrameBytes) fail(99, "frame larger than the emulator's records", -1);
}

inline void run_one(int tid) {
    Emu& E = emu();
    Rec& r = E.recs[tid];
    r.suspended = false;
    E.executions++;
#if defined(GTAP_FRAME_WORDS)
    int4 w[2];
    memcpy(w, r.frame, sizeof(w));
    __gtap_dispatch_words((unsigned long long)(void*)r.fn, r.frame, tid, nullptr, w[0], w[1]);
#elif defined(GTAP_DIRECT_DISPATCH)
    __gtap_dispatch((unsigned long long)(void*)r.fn, r.frame, tid, nullptr);
#else
    r.fn(r.frame, tid, nullptr);
#endif
    Rec& after = E.recs[tid];
    if (!after.finished && !after.suspended) fail(99, "an execution returned without finishing or suspending", tid);
    for (int c : E.staged) E.ready.push_back(c);
    E.staged.clear();
}

}  // namespace gtap_emu

// ---------------------------------------------------------------------------
// device ABI
// ---------------------------------------------------------------------------
inline int __gtap_get_task_state(int tid) {
#ifdef GTAP_ASSUME_NO_TASKWAIT
    (void)tid;
    return 0;
#else
    return gtap_emu::emu().recs[tid].state;
#endif
}

inline void* __gtap_spawn_task(TaskContext*, int self_tid, int* child_count, void (*func)(void*, int, TaskContext*),
                               int child_queue_idx, int* out_tid, bool retain_parent_result) {
    using namespace gtap_emu;
    Emu& E = emu();
    if (child_queue_idx < 0 || child_queue_idx >= GTAP_NUM_QUEUES) fail(1, "queue index out of range", self_tid);
    const int id = alloc_id();
    Rec& c = E.recs[id];
    c.fn = func;
    c.parent = self_tid;
#ifdef GTAP_ASSUME_NO_TASKWAIT
    c.retained = false;
    c.parent = -1;
    (void)retain_parent_result;
#else
    c.retained = retain_parent_result;
    E.recs[self_tid].pending++;
    E.recs[self_tid].since_join++;
#endif
    ++*child_count;
    E.staged.push_back(id);
    if (out_tid) *out_tid = id;
    return E.recs[id].frame;
}

inline bool __gtap_set_state_for_join(int tid, int child_count, int next_state, int queue_idx_after_join) {
    using namespace gtap_emu;
    Emu& E = emu();
    Rec& r = E.recs[tid];
    if (queue_idx_after_join < 0 || queue_idx_after_join >= GTAP_NUM_QUEUES) fail(2, "resume queue out of range", tid);
    if (child_count != r.since_join) fail(99, "join count differs from the children spawned since the last join", tid);
    r.since_join = 0;
    r.state = next_state;
    if (child_count == 0 || r.pending == 0) return false;
    r.suspended = true;
    return true;
}

inline void __gtap_finish_task(int tid, TaskContext*) {
    using namespace gtap_emu;
    Emu& E = emu();
    Rec& r = E.recs[tid];
    r.finished = true;
    if (r.pending > 0) {
        // children outstanding: they become orphans
        for (size_t i = 0; i < E.recs.size(); ++i)
            if (E.recs[i].live && E.recs[i].parent == tid) E.recs[i].parent = -1;
    }
    const int p = r.parent;
    if (p >= 0) {
        Rec& pr = E.recs[p];
        if (--pr.pending == 0 && pr.suspended) E.ready.push_back(p);
    }
    if (!r.retained) free_id(tid);
}

inline void* __gtap_get_task_data(int tid) { return gtap_emu::emu().recs[tid].frame; }

template <typename TaskType>
inline TaskType* __gtap_get_task_data(int tid) {
    return reinterpret_cast<TaskType*>(__gtap_get_task_data(tid));
}

inline void __gtap_release_task_id(int tid) {
    using namespace gtap_emu;
    Emu& E = emu();
    Rec& r = E.recs[tid];
    if (!r.live || !r.retained || !r.finished) {
        fail(99, "release of a task that is not a finished retained child", tid);
        return;
    }
    free_id(tid);
}

inline void __gtap_push_initial_task(void (*func)(void*, int, TaskContext*), int initial_queue_idx) {
    using namespace gtap_emu;
    Emu& E = emu();
    if (initial_queue_idx < 0 || initial_queue_idx >= GTAP_NUM_QUEUES) fail(1, "queue index out of range", 0);
    const int id = alloc_id();
    if (id != 0) fail(99, "the initial task is not task 0", id);
    E.recs[id].fn = func;
    E.ready.push_back(id);
}

inline void __gtap_execute_task_loop_device() {
    using namespace gtap_emu;
    Emu& E = emu();
    while (!E.ready.empty() && !E.error) {
        int tid;
        if (E.order == 0) {
            tid = E.ready.back();
            E.ready.pop_back();
        } else if (E.order == 1) {
            tid = E.ready.front();
            E.ready.pop_front();
        } else {
            const size_t i = (size_t)(E.rng() % E.ready.size());
            tid = E.ready[i];
            E.ready[i] = E.ready.back();   // any order among the rest: the next pick is random too
            E.ready.pop_back();
        }
        run_one(tid);
    }
    for (size_t i = 0; i < E.recs.size() && !E.error; ++i)
        if (E.recs[i].live && !E.recs[i].finished) fail(99, "a task never ran to its end", (int)i);
}

// ---------------------------------------------------------------------------
// host API
// ---------------------------------------------------------------------------
inline cudaError_t gtap_initialize() {
    gtap_emu::reset();
    return cudaSuccess;
}
inline cudaError_t gtap_reset() {
    gtap_emu::reset();
    return cudaSuccess;
}
inline cudaError_t gtap_synchronize() { return cudaSuccess; }
inline cudaError_t gtap_finalize() { return cudaSuccess; }
inline cudaError_t gtap_get_runtime_error_code(int* code) {
    *code = gtap_emu::emu().error;
    return cudaSuccess;
}
inline cudaError_t gtap_check_runtime_error() { return gtap_emu::emu().error ? 1 : cudaSuccess; }
