// gtap_thread.cuh -- drop-in for the reference's runtime/gtap_thread.cuh
// (thread-executed mode: one task = one CUDA thread).
//
// A program lowered to the reference's task ABI (the switch-statement state
// machines clang-gtap emits for `#pragma gtap task / taskwait / entry`)
// compiles against this header unchanged and runs on the B200 scheduler of
// this repository:
//
//   nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a \
//        -I include -DGTAP_GRID_SIZE=... -DGTAP_BLOCK_SIZE=... prog.cu \
//        -L gtap_b200 -lgtap_b200
//
// Device ABI (runtime/detail/thread/gtap_runtime_thread.cuh and
// gtap_thread_core.cuh in the reference), with the same names, signatures
// and contracts:
//   __gtap_get_task_state            :663      __gtap_set_state_for_join     :672
//   __gtap_spawn_task                :768      __gtap_finish_task            :733
//   __gtap_push_initial_task         :818      __gtap_execute_task_loop_device :1043
//   __gtap_get_child_task_id         :700      (legacy; records INVALID_TASKWAIT)
//   __gtap_release_task_id           core:159  __gtap_get_task_data          core:163-170
//   __gtap_append_result_handle ... __gtap_clear_result_handles   core:172-248 (legacy)
// Host API (gtap_runtime_thread.cuh:338-441, gtap_runtime_error.cuh:38-249):
//   gtap_initialize, gtap_finalize, gtap_reset, gtap_synchronize,
//   gtap_get_runtime_error_code, gtap_check_runtime_error,
//   gtap_get_runtime_error_string, gtap_visualize_profile (PROFILE builds).
//
// What differs from the reference runtime underneath: the scheduler is the
// one in gtap_b200/csrc/gtap_thread_sched.cuh (lock-free packed-word deques,
// batched steals, per-root termination, never traps).  Device errors are
// recorded (first one wins), every worker returns, and gtap_synchronize()
// prints the report; the CUDA context stays usable.  The arena is allocated
// by libgtap_b200.so, so programs link it.
//
// Configuration macros (reference runtime/detail/common/gtap_config.cuh:6-28,
// gtap_runtime_thread.cuh:10-24): GTAP_GRID_SIZE, GTAP_BLOCK_SIZE (multiple of
// 32, at most 512), GTAP_NUM_QUEUES (1..4), GTAP_MAX_CHILD_TASKS (children a
// task spawns at most), GTAP_MAX_TASKS_PER_WARP (task ids per warp, capped at
// 2^26 ids in all).  New ones: GTAP_DEQUE_CAPACITY (per warp and queue,
// power of two; tasks beyond it spill to a global queue),
// GTAP_LEGACY_RESULT_HANDLES (enables the legacy result-handle functions).
// GTAP_ASSUME_NO_TASKWAIT keeps its reference meaning: no task waits for its
// children, so children are not linked to their parent.
#pragma once

#include <cuda_runtime.h>
#include <stdio.h>

#include "gtap_types.h"
#include "../gtap_b200/csrc/gtap_thread_sched.cuh"
#include "gtap_device_util.cuh"

#ifndef GTAP_WARP_SIZE
#define GTAP_WARP_SIZE 32
#endif
#ifndef GTAP_GRID_SIZE
#define GTAP_GRID_SIZE 1024
#endif
#ifndef GTAP_BLOCK_SIZE
#define GTAP_BLOCK_SIZE 256
#endif
#ifndef GTAP_MAX_CHILD_TASKS
#define GTAP_MAX_CHILD_TASKS 32
#endif
#ifndef GTAP_NUM_QUEUES
#define GTAP_NUM_QUEUES 1
#endif
#ifndef GTAP_MAX_TASKS_PER_WARP
#define GTAP_MAX_TASKS_PER_WARP 20000
#endif
#ifndef GTAP_NUM_WARPS
#define GTAP_NUM_WARPS ((GTAP_BLOCK_SIZE + GTAP_WARP_SIZE - 1) / GTAP_WARP_SIZE)
#endif
#ifndef GTAP_DEQUE_CAPACITY
#define GTAP_DEQUE_CAPACITY 4096
#endif
#ifndef GTAP_RESULT_HANDLE_CAPACITY
#define GTAP_RESULT_HANDLE_CAPACITY 1000
#endif
#ifndef MAX_PROFILE_DATA
#define MAX_PROFILE_DATA 30000
#endif

static_assert(GTAP_BLOCK_SIZE % GTAP_WARP_SIZE == 0, "GTAP_BLOCK_SIZE must be a multiple of 32");
static_assert(GTAP_NUM_QUEUES >= 1 && GTAP_NUM_QUEUES <= gtap::kMaxQueues, "GTAP_NUM_QUEUES must be 1..4");

// libgtap_b200.so entry points used here (declared in gtap.h, which this
// header does not include: its C functions share names with the reference's
// host functions defined below).
extern "C" {
int gtap_default_config(gtap_config* cfg);
int gtap_external_initialize(const gtap_config* cfg, int32_t workers);
int gtap_external_prepare(void* arena_out, int64_t arena_bytes);
int gtap_external_finalize(void);
int gtap_external_error_code(int32_t* error_code);
int gtap_external_check(void);
const char* gtap_get_runtime_error_string(int error_code);
int gtap_visualize_profile(const char* app_name);
}

// The per-warp scheduler state task code receives and passes back; opaque.
struct TaskContext;

// Programs that define GTAP_DIRECT_DISPATCH before including this header
// provide __gtap_dispatch (gtap_b200.lower emits it): it compares the stored
// function pointer with each task function of the program and calls the match
// directly, so the task bodies are inlined into the worker loop instead of
// being reached by an indirect call (which cannot be inlined and saves its
// registers to the stack on every call).
#ifdef GTAP_DIRECT_DISPATCH
__device__ void __gtap_dispatch(unsigned long long fn, void* frame, int tid, TaskContext* ctx);
#endif
// Programs that define GTAP_FRAME_WORDS (gtap_b200.lower --results parent)
// provide __gtap_dispatch_words instead: the worker loads the first 16 or 32
// frame bytes with the task header, in one round trip, and hands them to the
// task, which then reads its frame from registers.
#ifdef GTAP_FRAME_WORDS
__device__ void __gtap_dispatch_words(unsigned long long fn, void* frame, int tid, TaskContext* ctx, int4 w0,
                                      int4 w1);
#endif

// Largest task frame in bytes, defined by the lowered program
// (reference runtime/detail/common/gtap_runtime_common.cuh:9).
extern const size_t __gtap_auto_task_data_size;

namespace gtap_dropin {

constexpr int kWarps = GTAP_NUM_WARPS;
// children staged per warp and round: every lane's children plus the parents
// its finishing children resume
constexpr int kSpawnCap = ((GTAP_WARP_SIZE * (GTAP_MAX_CHILD_TASKS + 1) + 63) / 64) * 64;
constexpr size_t kStagingInts = (size_t)GTAP_NUM_QUEUES * (kSpawnCap + gtap::kLocalCap);
constexpr size_t kStateBytes = (size_t)kWarps * sizeof(gtap::WarpShared);
constexpr size_t kStaticSmemLimit = 48 * 1024;
// staging buffers live in shared memory when they fit beside the warp state,
// else in the arena's global staging area
constexpr bool kStagingInSmem = kStateBytes + kWarps * kStagingInts * sizeof(int) <= kStaticSmemLimit;
constexpr size_t kSmemBytes = kStateBytes + (kStagingInSmem ? kWarps * kStagingInts * sizeof(int) : 0);
static_assert(kStateBytes <= kStaticSmemLimit,
              "GTAP_BLOCK_SIZE too large for the drop-in header: per-warp scheduler state must fit 48 KB of "
              "static shared memory (at most 512 threads per block)");

constexpr long long kWantIds = (long long)GTAP_GRID_SIZE * GTAP_NUM_WARPS * GTAP_MAX_TASKS_PER_WARP;
constexpr long long kTotalIds = kWantIds < (1ll << 26) ? (kWantIds < 4096 ? 4096 : kWantIds) : (1ll << 26);

static __shared__ __align__(16) unsigned char smem[kSmemBytes];
// arena descriptor of the current launch (written by gtap_initialize / gtap_reset)
static __constant__ gtap::Arena arena;
// global warp index of the thread that called __gtap_push_initial_task (-1 before)
static __device__ int initial_warp;

__device__ __forceinline__ gtap::WarpShared& warp_state() {
    return reinterpret_cast<gtap::WarpShared*>(smem)[threadIdx.x >> 5];
}

// Tasks are called through the function pointer __gtap_spawn_task stored.
struct Program {
#ifdef GTAP_FRAME_WORDS
    static constexpr bool kFrameWords = true;
#else
    static constexpr bool kFrameWords = false;
#endif
    static constexpr bool kFuncTable = true;
    static constexpr bool kJoinSum = false;   // every continuation runs as a task
    static constexpr bool kSubRounds = false; // one pass of task bodies per round
    __device__ static int root_kind(int) { return -1; }   // roots come from __gtap_push_initial_task only
    __device__ static bool root_args_ok(const gtap_root&) { return true; }
    __device__ static void init_root(const gtap::Arena&, const gtap_root&, void*) {}
    __device__ static void warp_leaves(const gtap::Arena&, gtap::WarpShared&, unsigned, int, const int4&,
                                       const int4&) {}
    __device__ static void exec(const gtap::Arena&, gtap::WarpShared& S, int, int tid, void* frame,
                                const int4& fw0, const int4& fw1, unsigned long long fn) {
    (void)fw0;
    (void)fw1;
#if defined(GTAP_FRAME_WORDS)
        __gtap_dispatch_words(fn, frame, tid, reinterpret_cast<TaskContext*>(&S), fw0, fw1);
#elif defined(GTAP_DIRECT_DISPATCH)
        __gtap_dispatch(fn, frame, tid, reinterpret_cast<TaskContext*>(&S));
#else
        using Fn = void (*)(void*, int, TaskContext*);
        reinterpret_cast<Fn>(fn)(frame, tid, reinterpret_cast<TaskContext*>(&S));
#endif
    }
};

inline cudaError_t to_cuda(int rc) {
    if (rc == 0) return cudaSuccess;
    if (rc < 0) return (cudaError_t)(-rc);
    return cudaErrorUnknown;   // a GTAP_ERROR_* code; gtap_check_runtime_error() prints it
}

inline cudaError_t prepare_launch() {
    gtap::Arena A;
    int rc = gtap_external_prepare(&A, (int64_t)sizeof(A));
    if (rc) return to_cuda(rc);
    const int none = -1;
    cudaError_t e = cudaMemcpyToSymbol(initial_warp, &none, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(arena, &A, sizeof(A));
}

}  // namespace gtap_dropin

// ---------------------------------------------------------------------------
// device ABI
// ---------------------------------------------------------------------------
__device__ __forceinline__ int __gtap_get_task_state(int tid) {
    (void)tid;
#ifdef GTAP_ASSUME_NO_TASKWAIT
    return 0;
#else
    return gtap::rt_state(gtap_dropin::warp_state());
#endif
}

__device__ __forceinline__ bool __gtap_set_state_for_join(int tid, int child_count, int next_state,
                                                          int queue_idx_after_join) {
    (void)tid;
    return gtap::rt_join(gtap_dropin::arena, gtap_dropin::warp_state(), child_count, next_state,
                         queue_idx_after_join);
}

// Legacy: child ids live in the lowered frames (reference :698-711).
__device__ __forceinline__ int __gtap_get_child_task_id(int parent_tid, int child_index) {
    GTAP_ERROR(gtap_dropin::arena, gtap::ERR_INVALID_TASKWAIT, parent_tid, -1, child_index, GTAP_MAX_CHILD_TASKS);
    return 0;
}

extern "C" __device__ __forceinline__ void __gtap_finish_task(int tid, TaskContext* ctx) {
    (void)tid;
    gtap::rt_finish(*reinterpret_cast<gtap::WarpShared*>(ctx));
}

extern "C" __device__ __forceinline__ void* __gtap_spawn_task(TaskContext* ctx, int self_tid, int* child_count,
                                                              void (*func)(void*, int, TaskContext*),
                                                              int child_queue_idx, int* out_tid,
                                                              bool retain_parent_result) {
    (void)self_tid;
    const gtap::Arena& A = gtap_dropin::arena;
    gtap::WarpShared& S = *reinterpret_cast<gtap::WarpShared*>(ctx);
    int id = -1;
#ifdef GTAP_ASSUME_NO_TASKWAIT
    (void)retain_parent_result;
    void* frame = gtap::rt_spawn(A, S, gtap::kKindIndirect, child_queue_idx, child_count, &id, false, true);
#else
    void* frame = gtap::rt_spawn(A, S, gtap::kKindIndirect, child_queue_idx, child_count, &id,
                                 retain_parent_result, false);
#endif
    if ((unsigned)id < (unsigned)A.total_ids) {
        A.funcs[id] = reinterpret_cast<void*>(func);
#ifdef GTAP_LEGACY_RESULT_HANDLES
        A.handle_meta[3 * id] = -1;
        A.handle_meta[3 * id + 1] = -1;
        A.handle_meta[3 * id + 2] = 0;
#endif
    }
    if (out_tid) *out_tid = id;
    return frame;
}

// Creates task 0 (its frame is __gtap_get_task_data(0), filled by the caller
// after this returns); the calling warp runs it first.
extern "C" __device__ __forceinline__ void __gtap_push_initial_task(void (*func)(void*, int, TaskContext*),
                                                                    int initial_queue_idx) {
    const gtap::Arena& A = gtap_dropin::arena;
    int q = initial_queue_idx;
    if ((unsigned)q >= (unsigned)A.num_queues) {
        GTAP_ERROR(A, gtap::ERR_INVALID_QUEUE_IDX, 0, q, q, A.num_queues);
        q = 0;
    }
    int4 hw;
    hw.x = (int)((unsigned)gtap::kKindIndirect << 16 | (unsigned)q << 24);
    hw.y = -1;   // no parent
    hw.z = 0;    // no children yet
    hw.w = 0;    // root slot 0
    *reinterpret_cast<int4*>(gtap::hdr_of(A, 0)) = hw;
    A.funcs[0] = reinterpret_cast<void*>(func);
#ifdef GTAP_LEGACY_RESULT_HANDLES
    A.handle_meta[0] = -1;
    A.handle_meta[1] = -1;
    A.handle_meta[2] = 0;
#endif
    gtap_dropin::initial_warp = (int)(blockIdx.x * gtap_dropin::kWarps + (threadIdx.x >> 5));
}

// Every thread of the launch enters; returns when the initial task and all
// its descendants have finished, or after a device error.
extern "C" __device__ __forceinline__ void __gtap_execute_task_loop_device() {
    using namespace gtap_dropin;
    const gtap::Arena& A = arena;
    const int wib = threadIdx.x >> 5;
    const int worker = (int)blockIdx.x * kWarps + wib;
    if (blockDim.x != GTAP_BLOCK_SIZE || worker >= A.num_workers) {
        // launched with another geometry than GTAP_GRID_SIZE x GTAP_BLOCK_SIZE
        if ((threadIdx.x & 31) == 0) GTAP_ERROR(A, gtap::ERR_INVALID_ARGUMENT, -1, -1, worker, A.num_workers);
        return;
    }
    __syncwarp();
    const int first = (gtap::ld_relaxed(&initial_warp) == worker) ? 0 : -1;
    int* sbuf;
    int* lstk;
    if (kStagingInSmem) {
        int* base = reinterpret_cast<int*>(smem + kStateBytes) + (size_t)wib * kStagingInts;
        sbuf = base;
        lstk = base + (size_t)GTAP_NUM_QUEUES * kSpawnCap;
    } else {
        int* base = A.staging + (size_t)worker * kStagingInts;
        sbuf = base;
        lstk = base + (size_t)GTAP_NUM_QUEUES * kSpawnCap;
    }
    gtap::thread_worker_run<Program, GTAP_NUM_QUEUES>(A, warp_state(), worker, sbuf, lstk, first);
}

extern "C" __device__ __forceinline__ void __gtap_release_task_id(int tid) {
    gtap::rt_release_id_dbg(gtap_dropin::arena, tid);
    gtap::rt_release_id(gtap_dropin::arena, gtap_dropin::warp_state(), tid);
}

__device__ __forceinline__ void* __gtap_get_task_data(int tid) { return gtap::frame_of(gtap_dropin::arena, tid); }

template <typename TaskType>
__device__ __forceinline__ TaskType* __gtap_get_task_data(int tid) {
    return reinterpret_cast<TaskType*>(__gtap_get_task_data(tid));
}

// Legacy linked result handles (reference gtap_thread_core.cuh:172-248).
// Available with -DGTAP_LEGACY_RESULT_HANDLES (each spawn then clears the
// child's list); otherwise a call records GTAP_ERROR_INVALID_TASKWAIT.
#ifdef GTAP_LEGACY_RESULT_HANDLES
extern "C" __device__ __forceinline__ void __gtap_append_result_handle(int parent_tid, int kind, int child_tid,
                                                                      void* lhs_addr) {
    const gtap::Arena& A = gtap_dropin::arena;
    const int slot = atomicAdd(A.handle_top, 1);
    if (slot >= A.handle_cap) {
        GTAP_ERROR(A, gtap::ERR_RESULT_HANDLE_OVERFLOW, parent_tid, -1, slot, A.handle_cap);
        return;
    }
    gtap_result_handle h;
    h.child_tid = child_tid;
    h.kind = kind;
    h.next = -1;
    h.pad = 0;
    h.lhs_addr = lhs_addr;
    A.handles[slot] = h;
    int* meta = A.handle_meta + 3 * parent_tid;   // begin, last, count: written by the parent's lane only
    if (meta[1] >= 0) A.handles[meta[1]].next = slot;
    else meta[0] = slot;
    meta[1] = slot;
    meta[2] += 1;
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_begin(int tid) {
    return gtap_dropin::arena.handle_meta[3 * tid];
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_count(int tid) {
    return gtap_dropin::arena.handle_meta[3 * tid + 2];
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_child_tid(int i) {
    return gtap_dropin::arena.handles[i].child_tid;
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_kind(int i) {
    return gtap_dropin::arena.handles[i].kind;
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_next(int i) {
    return gtap_dropin::arena.handles[i].next;
}
extern "C" __device__ __forceinline__ void* __gtap_get_result_handle_lhs_addr(int i) {
    return gtap_dropin::arena.handles[i].lhs_addr;
}
extern "C" __device__ __forceinline__ void __gtap_clear_result_handles(int tid) {
    int* meta = gtap_dropin::arena.handle_meta + 3 * tid;
    meta[0] = -1;
    meta[1] = -1;
    meta[2] = 0;
}
#else
#define GTAP_DROPIN_NO_HANDLES_(tid) \
    GTAP_ERROR(gtap_dropin::arena, gtap::ERR_INVALID_TASKWAIT, (tid), -1, 0, 0)
extern "C" __device__ __forceinline__ void __gtap_append_result_handle(int parent_tid, int, int, void*) {
    GTAP_DROPIN_NO_HANDLES_(parent_tid);
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_begin(int tid) {
    GTAP_DROPIN_NO_HANDLES_(tid);
    return -1;
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_count(int tid) {
    GTAP_DROPIN_NO_HANDLES_(tid);
    return 0;
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_child_tid(int) {
    GTAP_DROPIN_NO_HANDLES_(-1);
    return -1;
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_kind(int) {
    GTAP_DROPIN_NO_HANDLES_(-1);
    return 0;
}
extern "C" __device__ __forceinline__ int __gtap_get_result_handle_next(int) {
    GTAP_DROPIN_NO_HANDLES_(-1);
    return -1;
}
extern "C" __device__ __forceinline__ void* __gtap_get_result_handle_lhs_addr(int) {
    GTAP_DROPIN_NO_HANDLES_(-1);
    return nullptr;
}
extern "C" __device__ __forceinline__ void __gtap_clear_result_handles(int tid) { GTAP_DROPIN_NO_HANDLES_(tid); }
#endif

// ---------------------------------------------------------------------------
// host API (reference names and return types)
// ---------------------------------------------------------------------------
inline cudaError_t gtap_initialize() {
    gtap_config c;
    int rc = gtap_default_config(&c);
    if (rc) return gtap_dropin::to_cuda(rc);
    c.mode = GTAP_MODE_THREAD;
    c.grid = GTAP_GRID_SIZE;
    c.block = GTAP_BLOCK_SIZE;
    c.num_queues = GTAP_NUM_QUEUES;
    c.deque_capacity = GTAP_DEQUE_CAPACITY;
    c.spawn_capacity = gtap_dropin::kSpawnCap;
    c.total_ids = gtap_dropin::kTotalIds;
    const size_t frame = (__gtap_auto_task_data_size + 15) / 16 * 16;
    c.frame_bytes = (int32_t)(frame < 16 ? 16 : frame);
    c.result_handles = GTAP_RESULT_HANDLE_CAPACITY;
#ifdef PROFILE
    c.profile_samples = MAX_PROFILE_DATA;
#endif
    rc = gtap_external_initialize(&c, GTAP_GRID_SIZE * GTAP_NUM_WARPS);
    if (rc) return gtap_dropin::to_cuda(rc);
    return gtap_dropin::prepare_launch();
}

inline cudaError_t gtap_finalize() { return gtap_dropin::to_cuda(gtap_external_finalize()); }

// Ready the runtime for the next exec_kernel launch.
inline cudaError_t gtap_reset() { return gtap_dropin::prepare_launch(); }

inline cudaError_t gtap_get_runtime_error_code(int* error_code) {
    int32_t code = 0;
    int rc = gtap_external_error_code(&code);
    if (rc) return gtap_dropin::to_cuda(rc);
    if (error_code) *error_code = code;
    return cudaSuccess;
}

inline cudaError_t gtap_check_runtime_error() {
    gtap_external_check();
    return cudaSuccess;
}

inline cudaError_t gtap_synchronize() {
    cudaError_t st = cudaDeviceSynchronize();
    if (st != cudaSuccess) {
        printf("CUDA ERROR: %s\n", cudaGetErrorString(st));
        return st;
    }
    return gtap_check_runtime_error();
}
