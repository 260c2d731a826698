// gtap_device.cuh -- device primitives of the B200 GTaP runtime.
//
// Memory-model helpers (scoped PTX ld/st/atom), the shared arena layout, the
// first-error-wins status word, the lap-tagged MPMC ring used for the global
// overflow queue and the free task-id pool, and the per-worker lock-free
// deque with a packed (tag | bottom | top) control word.
//
// Reference correspondence (paths relative to the reference project root):
//   * load_L2 / store_L2 / atomicCAS_acquire  runtime/detail/common/gtap_runtime_common.cuh:89-185
//     -> ld/st .relaxed.gpu / .acquire.gpu / .release.gpu and atom.acq_rel.gpu below.
//   * error enum and report                     runtime/detail/common/gtap_runtime_error.cuh:7-30
//     -> gtap::Err and GtapErrorReport; the device never traps, it records the
//        first error, raises the abort flag and every worker returns.
//   * WarpTaskQueue {count, queue_lock, queue_head, queue[]}  runtime/detail/thread/gtap_runtime_thread.cuh:28-34
//     -> DequeCtl: one 64-bit word, no lock; see deque_* below.
//   * global MPMC queue (experimental GQ)       runtime/detail/experimental/thread/gtap_runtime_thread_gq.cuh:484-621
//     -> Ring: slots carry a lap tag so consumers never read an unwritten slot
//        and no in-order commit spin is needed.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gtap_types.h"
#include "gtap_ring.h"

namespace gtap {

constexpr int kWarp = 32;
constexpr int kMaxQueues = 4;
constexpr int kHdrBytes = 16;            // TaskHeader bytes in front of every frame
constexpr int kIdBits = 27;               // task ids are < 2^27
constexpr int kIdMask = (1 << kIdBits) - 1;

// Runtime error codes.  0..8 keep the reference's numbering
// (runtime/detail/common/gtap_runtime_error.cuh:7-18); the rest are new.
enum Err : int {
    ERR_NONE = GTAP_ERROR_NONE,
    ERR_INVALID_QUEUE_IDX = GTAP_ERROR_INVALID_QUEUE_IDX,
    ERR_INVALID_QUEUE_IDX_AFTER_JOIN = GTAP_ERROR_INVALID_QUEUE_IDX_AFTER_JOIN,
    ERR_QUEUE_OVERFLOW = GTAP_ERROR_QUEUE_OVERFLOW,
    ERR_RESULT_HANDLE_OVERFLOW = GTAP_ERROR_RESULT_HANDLE_OVERFLOW,
    ERR_POOL_SLOT_BUSY = GTAP_ERROR_TASK_ID_POOL_SLOT_BUSY,
    ERR_POOL_EXHAUSTED = GTAP_ERROR_TASK_ID_POOL_LOW_HEADROOM,
    ERR_SPAWN_BUFFER_OVERFLOW = GTAP_ERROR_GENERATED_TASK_ID_BUFFER_OVERFLOW,
    ERR_INVALID_TASKWAIT = GTAP_ERROR_INVALID_TASKWAIT,
    ERR_TIMEOUT = GTAP_ERROR_TIMEOUT,
    ERR_INVALID_KIND = GTAP_ERROR_INVALID_KIND,
    ERR_INVALID_ARGUMENT = GTAP_ERROR_INVALID_ARGUMENT,
};

// ---------------------------------------------------------------------------
// scoped memory operations
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ long long ld_relaxed(const long long* p) {
    long long v;
    asm volatile("ld.relaxed.gpu.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(int* p, int v) {
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(unsigned* p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(long long* p, long long v) {
    asm volatile("st.relaxed.gpu.global.s64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Task records are read with L1-bypassing vector loads: the data was written
// by another SM and published through a release/acquire pair.
__device__ __forceinline__ int4 ld_cg_v4(const void* p) {
    int4 v;
    asm volatile("ld.global.cg.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p) : "memory");
    return v;
}
// Loads of data written with plain stores (task records, sort buffers).
// Readers on the writer's SM see the writes through L1; readers on other SMs
// reach them only through an acquire (steal, pop, overflow ring, join), which
// also drops stale L1 lines.  GTAP_RECORD_LOAD selects the load flavour.
#ifndef GTAP_RECORD_LOAD
#define GTAP_RECORD_LOAD 1
#endif
// 16-byte asynchronous copy global -> shared through L2 (the path of ld.cg);
// both addresses 16-byte aligned.  rec_stage_wait: this thread's copies done.
__device__ __forceinline__ void cp_async16_cg(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void rec_stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ int4 ld_data_v4(const void* p) {
#if GTAP_RECORD_LOAD == 0
    int4 v;
    asm volatile("ld.global.cg.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p) : "memory");
    return v;
#else
    int4 v;
    asm volatile("ld.global.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p) : "memory");
    return v;
#endif
}
__device__ __forceinline__ unsigned long long ld_data_u64(const unsigned long long* p) {
    unsigned long long v;
#if GTAP_RECORD_LOAD == 0
    asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
#else
    asm volatile("ld.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
#endif
    return v;
}
__device__ __forceinline__ int ld_data(const int* p) {
    int v;
#if GTAP_RECORD_LOAD == 0
    asm volatile("ld.global.cg.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
#else
    asm volatile("ld.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
#endif
    return v;
}
__device__ __forceinline__ int ld_cg(const int* p) {
    int v;
    asm volatile("ld.global.cg.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int atom_add_acq_rel(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
// Acquire only: the caller has issued its own release fence before it.
__device__ __forceinline__ int atom_add_acquire(int* p, int v) {
    int old;
    asm volatile("atom.acquire.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ int atom_add_relaxed(int* p, int v) {
    int old;
    asm volatile("atom.relaxed.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned atom_add_relaxed(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.relaxed.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ long long atom_add_acq_rel(long long* p, long long v) {
    long long old;
    asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}
__device__ __forceinline__ void red_add_relaxed(long long* p, long long v) {
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_add_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_add_release(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_add_relaxed_i32(int* p, int v) {
    asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_add_release(int* p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long atom_cas_acquire(unsigned long long* p, unsigned long long cmp,
                                                               unsigned long long val) {
    unsigned long long old;
    asm volatile("atom.acquire.gpu.global.cas.b64 %0, [%1], %2, %3;"
                 : "=l"(old) : "l"(p), "l"(cmp), "l"(val) : "memory");
    return old;
}
__device__ __forceinline__ unsigned atom_cas_relaxed(unsigned* p, unsigned cmp, unsigned val) {
    unsigned old;
    asm volatile("atom.relaxed.gpu.global.cas.b32 %0, [%1], %2, %3;"
                 : "=r"(old) : "l"(p), "r"(cmp), "r"(val) : "memory");
    return old;
}
__device__ __forceinline__ int atom_cas_relaxed(int* p, int cmp, int val) {
    int old;
    asm volatile("atom.relaxed.gpu.global.cas.b32 %0, [%1], %2, %3;"
                 : "=r"(old) : "l"(p), "r"(cmp), "r"(val) : "memory");
    return old;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void fence_sc_sys() { asm volatile("fence.sc.sys;" ::: "memory"); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned lane_id() {
    unsigned l;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}
__device__ __forceinline__ unsigned smid() {
    unsigned s;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
    return s;
}

// ---------------------------------------------------------------------------
// Task record: 16-byte header followed by the frame
// ---------------------------------------------------------------------------
// Reference TaskHeader (runtime/detail/thread/gtap_thread_core.cuh:22-43) is
// 40 bytes in a separate array from the frames.  Here the header sits in the
// same 16-byte-aligned record as the frame so one vector load brings both.
// `generation`/`parent_generation` are not needed: a child whose parent
// returned without a taskwait is marked an orphan (parent = -1) at the end of
// the parent's execution, before the child can run.
struct TaskHeader {
    uint16_t state;   // resume label of the switch state machine (0 = fresh)
    uint8_t kind;     // task function index; kKindIndirect = use func table
    uint8_t flags;    // bits 0-2: spawn queue, bit 3: retain result for parent
    int32_t parent;   // parent tid, -1 for roots and orphans
    int32_t join;     // bits 0-23: children still outstanding; bits 24-26: resume queue;
                      // bit 27: the continuation only sums two int32 results (kJoinSumBit)
    int32_t root;     // root slot this task belongs to
};
static_assert(sizeof(TaskHeader) == kHdrBytes, "header must be 16 bytes");

constexpr uint8_t kFlagRetain = 0x8;
constexpr uint8_t kFlagJoinFinish = 0x10;   // block mode: after its taskwait the task only finishes
constexpr uint8_t kKindIndirect = 255;
constexpr int kJoinCountMask = 0x00FFFFFF;
// Thread mode: the task's code after its taskwait returns frame word 1 + frame
// word 2 (int32, wrapping) into its parent's frame at the byte offset in the
// low byte of frame word 3 (into the root's result for a root task) and
// finishes.  The child
// whose join decrement sees this bit with a count of one does exactly that in
// place of resuming the task, and goes on to the grandparent's join.
constexpr int kJoinSumBit = 1 << 27;

// ---------------------------------------------------------------------------
// MPMC ring of 32-bit values; each 64-bit slot = (lap + 1) << 32 | (value + 1)
// (encoding and its invariants: gtap_ring.h).  The cursors keep counting
// across launches; a launch starts with head moved to tail.
// ---------------------------------------------------------------------------
struct Ring {
    unsigned long long* slots;
    unsigned* head;       // consumer cursor
    unsigned* tail;       // producer cursor
    unsigned cap_log2;
};

// ---------------------------------------------------------------------------
// Arena: everything a launch needs, passed by value as the kernel parameter
// ---------------------------------------------------------------------------
struct Arena {
    // geometry
    int num_workers;        // warps (thread mode) or blocks (block mode)
    int warps_per_block;
    int num_queues;         // EPAQ queues (1..4)
    int deque_cap_log2;     // ring capacity per worker per queue
    int steal_batch;        // max tasks moved by one steal
    int victim_policy;      // GTAP_VICTIM_*
    int probe_width;        // victims probed per steal attempt (thread mode)
    int spawn_cap;          // staged children per queue per worker and round
    int ids_per_worker;     // private initial id range per worker
    int avail_target;       // most free ids a worker keeps cached (<= 224)
    int rec_stride;         // bytes per task record
    int admit_batch;        // roots claimed per admission
    int mode;               // GTAP_MODE_*
    int id_base;            // first id of the private ranges (ids below it are reserved)
    int publish_lazy;       // 0 or 1 for this launch (gtap_config::publish_lazy)
    int join_walk;          // rounds of at most this many tasks run fib sums at their joins (gtap_config::join_walk)
    int sub_rounds;         // extra passes of task bodies on a round's idle lanes (gtap_config::sub_rounds)
    int max_inflight;       // admitted-but-unfinished roots allowed (0 = unlimited)
    int total_ids;          // ids in the arena
    unsigned long long watchdog_ns;
    unsigned long long t0_ns;

    // task storage
    char* records;                     // [total_ids][rec_stride]
    void** funcs;                      // [total_ids] for kKindIndirect tasks (may be null)

    // deques
    unsigned long long* dq_ctl;        // [Q][W]
    int* dq_slots;                     // [Q][W][cap]

    // global queues
    Ring overflow;                     // task ids that did not fit a deque
    Ring idpool;                       // recycled task ids
    unsigned* fresh_next;              // next never-used id beyond the private ranges

    // roots
    const gtap_root* roots;            // root descriptors
    gtap_root_result* results;         // per root
    long long* outstanding;            // per root: pre-charged outstanding count
    int n_roots;                       // batch: roots in the table; serve: ring capacity
    unsigned* next_root;               // admission cursor
    const unsigned* published;         // serve: roots published by the host (device memory)
    const int* shutdown;               // serve: host asks the kernel to drain and exit
    unsigned* completed;               // roots completed
    unsigned long long* done_ring;     // serve: completion ring (host-mapped), entries = root index + 1
    unsigned done_ring_cap;
    int* live_tasks;                   // tasks created and not finished (admission watermark)
    int admit_watermark;               // serve: admit while live_tasks < watermark

    // status
    int* status;                       // first error code
    int* abort_flag;
    int* done_flag;
    GtapErrorReport* report;           // host-mapped report (may be null)

    // debug builds (GTAP_DEBUG_IDS): live flag and fresh-execution flag per id
    int* dbg_live;
    int* dbg_exec;
    unsigned* dbg_slotpos;   // position each deque slot was last written for

    // count of idle workers, replicated (see kHungryReplicas); busy workers
    // publish part of their local work while it is non-zero
    int* hungry;

    // statistics: [W][GTAP_STAT_COUNT]
    unsigned long long* stats;

    // profiling timelines (reference gtap_profile_thread.cuh:29-108, 188-268)
    long long* prof_having;            // [W][prof_cap]
    long long* prof_working;           // [W][prof_cap]
    int* prof_tasks;                   // [W][prof_cap]
    int prof_cap;                      // 0 = profiling off

    // legacy result-handle table (reference gtap_thread_core.cuh:172-248)
    gtap_result_handle* handles;
    int* handle_top;
    int* handle_meta;                  // [total_ids][3]: begin, last, count

    // kernels launched by the caller (drop-in header) whose per-warp staging
    // buffers do not fit static shared memory: [workers][Q][spawn_cap + kLocalCap]
    int* staging;
    int handle_cap;
    int leaf_buf;                      // leaf input buffers per warp at the end of dynamic shared memory (0: none)
    int rec_prefetch;                  // 1: the kernel's dynamic shared memory holds a record stage per warp
                                       //    (kRecStageBytes; the leaf buffers double as it where there are any)
};

// ---------------------------------------------------------------------------
// status / errors: first error wins, never trap
// ---------------------------------------------------------------------------
static __device__ __noinline__ void record_error(const Arena& A, int code, int tid, int queue_idx, int value, int limit,
                                          int line) {
    if (atomicCAS(A.status, 0, code) == 0) {
        GtapErrorReport* r = A.report;
        if (r) {
            r->code = code;
            r->src_line = line;
            r->block_idx = blockIdx.x;
            r->thread_idx = threadIdx.x;
            r->tid = tid;
            r->queue_idx = queue_idx;
            r->value = value;
            r->limit = limit;
            __threadfence_system();
            r->valid = 1;
            __threadfence_system();
        }
    }
    atomicExch(A.abort_flag, 1);
}
#define GTAP_ERROR(A, code, tid, q, value, limit) ::gtap::record_error((A), (code), (tid), (q), (value), (limit), __LINE__)

__device__ __forceinline__ bool aborted(const Arena& A) { return ld_relaxed(A.abort_flag) != 0; }

// ---------------------------------------------------------------------------
// Ring operations (warp-cooperative; all lanes of the warp call them)
// ---------------------------------------------------------------------------
// Push n values held by lanes [0, n).  Both global rings are sized to hold
// every task id of the arena, and every value pushed is a distinct live id, so
// a reservation by atomicAdd can never overrun unconsumed slots.  Values must
// be published already (the caller issues its release fence before the push).
static __device__ void ring_push_warp(const Arena& A, const Ring& r, int value, int n) {
    const unsigned lane = lane_id();
    const unsigned cap = 1u << r.cap_log2;
    unsigned pos = 0;
    if (lane == 0) pos = atom_add_relaxed(r.tail, (unsigned)n);
    pos = __shfl_sync(0xffffffffu, pos, 0);
    (void)A;
    if ((int)lane < n) {
        unsigned p = pos + lane;
        st_relaxed(&r.slots[p & (cap - 1)], (unsigned long long)ring_word_of(p, r.cap_log2, value));
    }
}

// single-lane push (slow paths)
__device__ __forceinline__ void ring_push_one(const Ring& r, int value) {
    const unsigned cap = 1u << r.cap_log2;
    unsigned p = atom_add_relaxed(r.tail, 1u);
    st_relaxed(&r.slots[p & (cap - 1)], (unsigned long long)ring_word_of(p, r.cap_log2, value));
}

// Claims for the recycled-id pool (one thread).  Many warps refill their id
// caches at the same moments (a wave of spawns), and a claim by
// compare-and-swap on the consumer cursor then fails for all but one of them
// per round trip: measured on B200 with cilksort roots, ~49 attempts of ~8k
// cycles per claim.  While the pool is long, one atomic add claims instead;
// it cannot fail.  Positions it claims past the producer cursor (possible
// only when other claims overtook this one) are given up: their ids, written
// there later, are simply never handed out again in this launch -- the pool
// holds interchangeable free ids, and the next launch starts with every id
// free again.  Returns the number of positions from *pos that hold produced
// values.
constexpr unsigned kPoolFaaMargin = 4096;   // pool length above which claims use the atomic add
__device__ __forceinline__ unsigned pool_claim(const Ring& r, unsigned want, unsigned& pos) {
    const unsigned cap = 1u << r.cap_log2;
    unsigned h = ld_relaxed(r.head);   // head first: then h <= t below
    unsigned t = ld_relaxed(r.tail);
    unsigned avail = t - h;
    if (avail == 0 || avail > cap) return 0;
    if (avail >= want + kPoolFaaMargin) {
        const unsigned p = atom_add_relaxed(r.head, want);
        const int produced = (int)(ld_relaxed(r.tail) - p);   // negative if other claims overtook this one
        pos = p;
        return produced <= 0 ? 0u : (produced < (int)want ? (unsigned)produced : want);
    }
    for (int attempt = 0; attempt < 64; ++attempt) {
        const unsigned k = avail < want ? avail : want;
        if (atom_cas_relaxed(r.head, h, h + k) == h) {
            pos = h;
            return k;
        }
        h = ld_relaxed(r.head);
        t = ld_relaxed(r.tail);
        avail = t - h;
        if (avail == 0 || avail > cap) return 0;
    }
    return 0;
}

// Pop up to `want` values into lanes [0, got).  Slots reserved by a producer
// but not yet written are waited for with a bounded spin.  pool: the ring is
// the recycled-id pool (claims by pool_claim).
static __device__ int ring_pop_warp(const Arena& A, const Ring& r, int want, int* value, bool pool = false) {
    const unsigned lane = lane_id();
    const unsigned cap = 1u << r.cap_log2;
    unsigned pos = 0;
    int got = 0;
    if (lane == 0 && pool) {
        got = (int)pool_claim(r, (unsigned)want, pos);
    } else if (lane == 0) {
        for (int attempt = 0; attempt < 64; ++attempt) {
            unsigned h = ld_relaxed(r.head);   // head first: then h <= t below
            unsigned t = ld_relaxed(r.tail);
            unsigned avail = t - h;
            if (avail == 0 || avail > cap) break;
            unsigned k = avail < (unsigned)want ? avail : (unsigned)want;
            if (atom_cas_relaxed(r.head, h, h + k) == h) { pos = h; got = (int)k; break; }
        }
    }
    got = __shfl_sync(0xffffffffu, got, 0);
    pos = __shfl_sync(0xffffffffu, pos, 0);
    if ((int)lane < got) {
        unsigned p = pos + lane;
        unsigned long long w = 0;
        int spins = 0;
        for (;;) {
            w = ld_acquire(&r.slots[p & (cap - 1)]);
            if (ring_word_ready(w, p, r.cap_log2)) break;
            if (++spins > (1 << 20)) {
                GTAP_ERROR(A, ERR_TIMEOUT, -1, -1, (int)p, 0);
                w = 0;
                break;
            }
            __nanosleep(64);
        }
        *value = ring_word_value(w);
    }
    return got;
}

// ---------------------------------------------------------------------------
// Deque control word: [tag:22 | bottom:21 | top:21]
// ---------------------------------------------------------------------------
constexpr int kPosBits = 21;
constexpr unsigned kPosMask = (1u << kPosBits) - 1;
__device__ __forceinline__ unsigned dq_top(unsigned long long w) { return (unsigned)(w & kPosMask); }
__device__ __forceinline__ unsigned dq_bottom(unsigned long long w) { return (unsigned)((w >> kPosBits) & kPosMask); }
__device__ __forceinline__ unsigned dq_size(unsigned long long w) { return (dq_bottom(w) - dq_top(w)) & kPosMask; }
__device__ __forceinline__ unsigned long long dq_with_top(unsigned long long w, unsigned top) {
    return (w & ~(unsigned long long)kPosMask) | (top & kPosMask);
}
__device__ __forceinline__ unsigned long long dq_owner_pop(unsigned long long w, unsigned k) {
    unsigned long long tag = (w >> (2 * kPosBits)) + 1;
    unsigned b = (dq_bottom(w) - k) & kPosMask;
    return (tag << (2 * kPosBits)) | ((unsigned long long)b << kPosBits) | dq_top(w);
}

__device__ __forceinline__ unsigned long long* dq_ctl_ptr(const Arena& A, int q, int w) {
    return A.dq_ctl + (size_t)q * A.num_workers + w;
}
__device__ __forceinline__ int* dq_slot_ptr(const Arena& A, int q, int w, unsigned pos) {
    return A.dq_slots + (((size_t)q * A.num_workers + w) << A.deque_cap_log2) + (pos & ((1u << A.deque_cap_log2) - 1));
}

__device__ __forceinline__ TaskHeader* hdr_of(const Arena& A, int tid) {
    return reinterpret_cast<TaskHeader*>(A.records + (size_t)tid * A.rec_stride);
}
__device__ __forceinline__ void* frame_of(const Arena& A, int tid) {
    return A.records + (size_t)tid * A.rec_stride + kHdrBytes;
}

}  // namespace gtap
