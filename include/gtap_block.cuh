// gtap_block.cuh -- drop-in for the reference's runtime/gtap_block.cuh
// (block-cooperative mode: one task = one CUDA block).
//
// A program lowered to the reference's block-mode task ABI compiles against
// this header unchanged and runs on the block scheduler of this repository
// (gtap_b200/csrc/gtap_block_sched.cuh):
//
//   nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a \
//        -I include -DGTAP_GRID_SIZE=... -DGTAP_BLOCK_SIZE=... prog.cu \
//        -L gtap_b200 -lgtap_b200
//
// Device ABI (reference runtime/detail/block/gtap_runtime_block.cuh and
// gtap_block_core.cuh), same names, signatures and contracts:
//   __gtap_get_task_state              :481      __gtap_set_state_for_join        :440
//   __gtap_set_state_for_join_block    :458      __gtap_spawn_task                :542
//   __gtap_finish_task                 :516      __gtap_push_initial_task         :577
//   __gtap_execute_task_loop_device    :770      __gtap_get_child_task_id         :489 (legacy)
//   __gtap_release_task_id             core:128  __gtap_get_task_data             core:131-139
// Every thread of the block runs the task body; any thread may spawn.  A
// taskwait joins the children the block spawned since the previous one
// (reference: ctx->task_id_generated_count).
// Host API (gtap_runtime_block.cuh:41-297, gtap_runtime_error.cuh:38-249):
//   gtap_initialize, gtap_finalize, gtap_reset, gtap_synchronize,
//   gtap_get_runtime_error_code, gtap_check_runtime_error,
//   gtap_get_runtime_error_string.
//
// Configuration macros: GTAP_GRID_SIZE (blocks), GTAP_BLOCK_SIZE (multiple of
// 32, at most 512), GTAP_MAX_TASKS_PER_BLOCK (task ids per block, capped at
// 2^26 ids in all), GTAP_DEQUE_CAPACITY (per block, power of two; tasks beyond
// it spill to a global queue).  GTAP_ASSUME_NO_TASKWAIT keeps its reference
// meaning: children are not linked to their parent.
#pragma once

#include <cuda_runtime.h>
#include <stdio.h>

#include "gtap_types.h"
#include "../gtap_b200/csrc/gtap_block_sched.cuh"
#include "gtap_device_util.cuh"

#ifndef GTAP_GRID_SIZE
#define GTAP_GRID_SIZE 592
#endif
#ifndef GTAP_BLOCK_SIZE
#define GTAP_BLOCK_SIZE 256
#endif
#ifndef GTAP_MAX_TASKS_PER_BLOCK
#define GTAP_MAX_TASKS_PER_BLOCK 10000
#endif
#ifndef GTAP_DEQUE_CAPACITY
#define GTAP_DEQUE_CAPACITY 4096
#endif
#ifndef GTAP_MAX_CHILD_TASKS
#define GTAP_MAX_CHILD_TASKS 32
#endif

static_assert(GTAP_BLOCK_SIZE % 32 == 0, "GTAP_BLOCK_SIZE must be a multiple of 32");
static_assert(GTAP_BLOCK_SIZE <= gtap::kBMaxThreads, "GTAP_BLOCK_SIZE must be at most 512 in block mode");

extern "C" {
int gtap_default_config(gtap_config* cfg);
int gtap_external_initialize(const gtap_config* cfg, int32_t workers);
int gtap_external_prepare(void* arena_out, int64_t arena_bytes);
int gtap_external_finalize(void);
int gtap_external_error_code(int32_t* error_code);
int gtap_external_check(void);
const char* gtap_get_runtime_error_string(int error_code);
}

// The per-block scheduler state task code receives and passes back; opaque.
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

// Largest task frame in bytes, defined by the lowered program
// (reference runtime/detail/common/gtap_runtime_common.cuh:9).
extern const size_t __gtap_auto_task_data_size;

namespace gtap_dropin {

constexpr long long kWantIds = (long long)GTAP_GRID_SIZE * GTAP_MAX_TASKS_PER_BLOCK;
constexpr long long kTotalIds = kWantIds < (1ll << 26) ? (kWantIds < 4096 ? 4096 : kWantIds) : (1ll << 26);

static __shared__ gtap::BlockShared block_state;
// arena descriptor of the current launch (written by gtap_initialize / gtap_reset)
static __constant__ gtap::Arena arena;
// block that called __gtap_push_initial_task (-1 before)
static __device__ int initial_block;

__device__ __forceinline__ gtap::BlockShared& state() { return block_state; }

// Tasks are called through the function pointer __gtap_spawn_task stored.
struct Program {
    static constexpr int kSmemInts = 0;
    static constexpr bool kFuncTable = true;
    __device__ static int root_kind(int) { return -1; }   // the root comes from __gtap_push_initial_task only
    __device__ static bool root_args_ok(const gtap_root&) { return true; }
    __device__ static void init_root(const gtap::Arena&, const gtap_root&, void*) {}
    __device__ static void exec(const gtap::Arena& A, gtap::BlockShared& S, int tid, int*) {
#ifdef GTAP_DIRECT_DISPATCH
        __gtap_dispatch(S.fn, gtap::frame_of(A, tid), tid, reinterpret_cast<TaskContext*>(&S));
#else
        using Fn = void (*)(void*, int, TaskContext*);
        reinterpret_cast<Fn>(S.fn)(gtap::frame_of(A, tid), tid, reinterpret_cast<TaskContext*>(&S));
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
    cudaError_t e = cudaMemcpyToSymbol(initial_block, &none, sizeof(int));
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
    return gtap::bt_state(gtap_dropin::state());
#endif
}

// taskwait (reference :458-479): every thread of the block calls it; true if
// the task suspends until the children spawned since the last taskwait finish.
extern "C" __device__ __forceinline__ bool __gtap_set_state_for_join_block(int tid, TaskContext* ctx, int next_state,
                                                                         int unused_value) {
    (void)tid;
    (void)unused_value;
    return gtap::bt_join(gtap_dropin::arena, *reinterpret_cast<gtap::BlockShared*>(ctx), next_state);
}

// The thread-mode signature, kept by the reference's block runtime
// (:440-456); the join count is the block's, as in the _block variant.
extern "C" __device__ __forceinline__ bool __gtap_set_state_for_join(int tid, int child_count, int next_state,
                                                                   int unused_value) {
    (void)tid;
    (void)child_count;
    (void)unused_value;
    return gtap::bt_join(gtap_dropin::arena, gtap_dropin::state(), next_state);
}

// Legacy: child ids live in the lowered frames (reference :489-499).
__device__ __forceinline__ int __gtap_get_child_task_id(int parent_tid, int child_index) {
    GTAP_ERROR(gtap_dropin::arena, gtap::ERR_INVALID_TASKWAIT, parent_tid, -1, child_index, GTAP_MAX_CHILD_TASKS);
    return 0;
}

extern "C" __device__ __forceinline__ void __gtap_finish_task(int tid, TaskContext* ctx) {
    (void)tid;
    gtap::bt_finish(*reinterpret_cast<gtap::BlockShared*>(ctx));
}

// Any thread of the block (reference :542-575).
extern "C" __device__ __forceinline__ void* __gtap_spawn_task(TaskContext* ctx, int self_tid, int* child_count,
                                                              void (*func)(void*, int, TaskContext*),
                                                              int unused_value, int* out_tid,
                                                              bool retain_parent_result) {
    (void)self_tid;
    (void)unused_value;
    const gtap::Arena& A = gtap_dropin::arena;
    gtap::BlockShared& S = *reinterpret_cast<gtap::BlockShared*>(ctx);
    int id = -1;
#ifdef GTAP_ASSUME_NO_TASKWAIT
    (void)retain_parent_result;
    void* frame = gtap::bt_spawn(A, S, gtap::kKindIndirect, child_count, &id, false, true);
#else
    void* frame = gtap::bt_spawn(A, S, gtap::kKindIndirect, child_count, &id, retain_parent_result, false);
#endif
    if ((unsigned)id < (unsigned)A.total_ids) A.funcs[id] = reinterpret_cast<void*>(func);
    if (out_tid) *out_tid = id;
    return frame;
}

// Creates task 0 (its frame is __gtap_get_task_data(0), filled by the caller
// after this returns); the calling block runs it first.
extern "C" __device__ __forceinline__ void __gtap_push_initial_task(void (*func)(void*, int, TaskContext*),
                                                                    int unused_value) {
    (void)unused_value;
    const gtap::Arena& A = gtap_dropin::arena;
    int4 hw;
    hw.x = (int)((unsigned)gtap::kKindIndirect << 16);
    hw.y = -1;   // no parent
    hw.z = 0;    // no children yet
    hw.w = 0;    // root slot 0
    *reinterpret_cast<int4*>(gtap::hdr_of(A, 0)) = hw;
    A.funcs[0] = reinterpret_cast<void*>(func);
    gtap_dropin::initial_block = (int)blockIdx.x;
}

// Every thread of the launch enters; returns when the initial task and all
// its descendants have finished, or after a device error.
extern "C" __device__ __forceinline__ void __gtap_execute_task_loop_device() {
    using namespace gtap_dropin;
    const gtap::Arena& A = arena;
    if (blockDim.x != GTAP_BLOCK_SIZE || (int)blockIdx.x >= A.num_workers) {
        // launched with another geometry than GTAP_GRID_SIZE x GTAP_BLOCK_SIZE
        if (threadIdx.x == 0) GTAP_ERROR(A, gtap::ERR_INVALID_ARGUMENT, -1, -1, (int)blockIdx.x, A.num_workers);
        return;
    }
    __syncthreads();   // the initial task's frame is written before the loop reads it
    const int first = (gtap::ld_relaxed(&initial_block) == (int)blockIdx.x) ? 0 : -1;
    gtap::block_worker<Program>(A, state(), nullptr, first);
}

// A retained child's id, once the task has read its frame (reference
// gtap_block_core.cuh:128-131); any thread, returned after the body.
extern "C" __device__ __forceinline__ void __gtap_release_task_id(int tid) {
    gtap::bt_release_deferred(gtap_dropin::arena, gtap_dropin::state(), tid);
}

__device__ __forceinline__ void* __gtap_get_task_data(int tid) { return gtap::frame_of(gtap_dropin::arena, tid); }

template <typename TaskType>
__device__ __forceinline__ TaskType* __gtap_get_task_data(int tid) {
    return reinterpret_cast<TaskType*>(__gtap_get_task_data(tid));
}

// ---------------------------------------------------------------------------
// host API (reference names and return types)
// ---------------------------------------------------------------------------
inline cudaError_t gtap_initialize() {
    gtap_config c;
    int rc = gtap_default_config(&c);
    if (rc) return gtap_dropin::to_cuda(rc);
    c.mode = GTAP_MODE_BLOCK;
    c.grid = GTAP_GRID_SIZE;
    c.block = GTAP_BLOCK_SIZE;
    c.num_queues = 1;
    c.deque_capacity = GTAP_DEQUE_CAPACITY;
    c.total_ids = gtap_dropin::kTotalIds;
    const size_t frame = (__gtap_auto_task_data_size + 15) / 16 * 16;
    c.frame_bytes = (int32_t)(frame < 16 ? 16 : frame);
    rc = gtap_external_initialize(&c, GTAP_GRID_SIZE);
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
