// gtap_thread_sched.cuh -- thread-executed mode: one task per CUDA thread,
// one worker per warp, persistent kernel.
//
// Reference: runtime/detail/thread/gtap_runtime_thread.cuh (paths relative to
// the reference project root).
//   __gtap_execute_task_loop_device_impl :849-1040  -> worker_loop()
//   pop_batch :511-536                              -> pop_own()
//   steal_batch :538-593                            -> steal()
//   push_batch :595-660                             -> finish_round() (select + publish)
//   reserve_unpublished_task_id :38-48              -> stage_child()
//   __gtap_spawn_task :768-816                      -> rt_spawn()
//   __gtap_set_state_for_join :672-696              -> rt_join()
//   __gtap_finish_task / notify_parent :714-764     -> rt_finish() + finish_round()
//   get_task_id_from_warp_pool / release :111-146 (gtap_thread_core.cuh) -> id cache below
//   termination :927-964                            -> per-root balances (no active-worker counter)
//
// Differences that matter for speed on B200:
//   * the up-to-32 tasks a warp runs next stay in registers; only the surplus
//     is written to the deque and published with ONE release add per queue;
//   * no victim lock: steals claim a batch with one CAS on a packed
//     (tag | bottom | top) word, and up to probe_width victims are probed in
//     parallel by different lanes before choosing the fullest;
//   * no __threadfence() per task: a finishing child performs one acq_rel
//     decrement of the parent's join word, which also carries the queue the
//     parent resumes on;
//   * task ids come from a per-warp shared-memory cache refilled in batches of
//     32 (private range, then the global recycled-id ring, then fresh ids);
//   * termination: each warp holds pre-charged per-root balances, so the
//     global per-root counter is touched once per ~kBalChunk tasks and a root
//     completes exactly when its counter returns to zero.
#pragma once
#include "gtap_device.cuh"

namespace gtap {

// Profiling builds (-DGTAP_PHASE_TIMERS): lane 0 adds the clock64 cycles of
// each scheduler phase to statistics slots 10..15 (acquire, load + task
// bodies, warp leaves + orphans + staging of children and deque slots, fence
// + publication + joins + id release + resumed parents, root accounting, id
// cache).  Off by default: the timers cost a few instructions per phase.
#ifdef GTAP_PHASE_TIMERS
// slot 9 (overflow pushes) holds the task-record load latency and slot 7
// (published) the publication fence in these builds
#define GTAP_PHASE_MARK(t) long long t = clock64()
#define GTAP_PHASE_MARK_AFTER(t, dep) \
    long long t;                      \
    asm volatile("mov.u64 %0, %%clock64;" : "=l"(t) : "r"(dep) : "memory")
#define GTAP_PHASE_ADD(slot, t0, t1) \
    do {                                 \
        if (lane_id() == 0) S.st[slot] += (unsigned long long)((t1) - (t0)); \
    } while (0)
#else
#define GTAP_PHASE_MARK_AFTER(t, dep) (void)0
#define GTAP_PHASE_MARK(t) (void)0
#define GTAP_PHASE_ADD(slot, t0, t1) (void)0
#endif

constexpr int kAvailCap = 256;    // per-warp cache of free task ids (a ring; power of two)
constexpr int kAvailHigh = 240;   // above this, 32 ids go back to the recycled pool
constexpr int kFreedCap = 96;
constexpr int kRootBalCap = 8;
constexpr int kBalChunk = 1024;
constexpr int kLocalCap = 128;     // per-warp, per-queue local ready stack (power of two)
// Per-warp record stage: each lane's next task record (header and up to 32
// frame bytes), copied in while the previous round ends.
constexpr int kRecStageBytes = kWarp * 48;
constexpr int kReserve = 32;       // ready tasks a warp keeps when others are hungry
constexpr int kHungryReplicas = 8;  // copies of the hungry-worker count, 128 bytes apart
constexpr int kHungryStride = 32;

// l_flags bits: each lane writes only its own entry, the round end reads them
// back with ballots (no shared-memory atomics on one word from 32 lanes)
constexpr int kLaneFinished = 1;   // the task returned (rt_finish)
constexpr int kLaneRetain = 2;     // ... and its parent reads its frame, so the parent releases the id
constexpr int kLaneLeaf = 4;       // the task left leaf work for the whole warp (warp_leaves)

struct RootBal {
    int root;
    int bal;
    int created;
    int touched;
};

// Per-warp shared state.  This is the object the task ABI calls TaskContext.
struct WarpShared {
    int l_tid[kWarp];
    int l_root[kWarp];
    unsigned l_w0[kWarp];      // header word 0 of the running task: state | kind << 16 | flags << 24
    int l_parent[kWarp];
    int l_spawned[kWarp];      // children spawned since the last taskwait
    int l_created[kWarp];      // tasks this lane created this round
    int l_value[kWarp];        // contributions to the lane's root value (n-queens counts)
    int l_flags[kWarp];        // this round, per lane: kLaneFinished | kLaneRetain | kLaneLeaf
    int l_pend[kWarp];         // detached child past the staging buffer whose frame is still being written (-1: none)
    int cnt[kMaxQueues];       // children staged this round, per queue
    int avail_n, alloc_pos, freed_n, bump;
    int avail_head;            // avail[] is a ring: the next free id is avail[avail_head]
    int alloc_last;            // ids this warp allocated last round (refill target)
    int avail[kAvailCap];
    int freed[kFreedCap];
    int nbal;
    RootBal bal[kRootBalCap];
    unsigned long long st[GTAP_STAT_COUNT];
    int worker;
    int prof_h, prof_w;
    unsigned seen_done;        // watchdog (lane 0): completions seen at t_watch
    unsigned long long t_watch;
    int* sbuf;                 // [num_queues][spawn_cap] staged child ids (| spawner lane << 27)
    int* lstk;                 // [num_queues][kLocalCap] ready tasks not yet visible to thieves
    int* lbuf;                 // leaf buffers: [A.leaf_buf + 1][Prog::kLeafKeys] (programs with warp leaves), or null
    int4* rstage;              // record stage [kWarp][3] (kRecStageBytes), or null: records are loaded when a round starts
};

// Positions of this warp's local stacks and deques.  Only the scheduler
// changes them, identically in every lane: each lane keeps its own copy, so
// no lane waits for another to publish an update through shared memory.
// QM: the most queues the kernel supports (1 or kMaxQueues); fewer entries
// fewer registers.
template <int QM>
struct QueuePos {
    unsigned ls_lo[QM];      // local stack: oldest entry (published first)
    unsigned ls_hi[QM];      // local stack: one past the newest entry (run first)
    unsigned bottom[QM];     // deque bottom, entries staged this round included
    unsigned top_cache[QM];  // deque top last read (it only grows)
    int pend[QM];            // deque entries staged this round, not yet published
    int cur_q;               // EPAQ queue to try first (reference ctx->queue_idx)
};

// Element k of a per-queue array through constant indices only, so that
// QueuePos stays in registers instead of local memory.
template <class T, int N>
__device__ __forceinline__ T qget(const T (&a)[N], int k) {
    T v = a[0];
#pragma unroll
    for (int i = 1; i < N; ++i)
        if (k == i) v = a[i];
    return v;
}
template <class T>
struct QNoDeduce {
    using type = T;
};
template <class T, int N>
__device__ __forceinline__ void qset(T (&a)[N], int k, typename QNoDeduce<T>::type v) {
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (k == i) a[i] = v;
}

// The queues a kernel serves: a kernel built for one queue (QM == 1) only
// runs launches with one, so the count folds to a constant there.
template <int QM>
__device__ __forceinline__ int queue_count(const Arena& A) {
    return QM == 1 ? 1 : A.num_queues;
}

template <int QM>
__device__ __forceinline__ void queue_pos_init(QueuePos<QM>& P) {
#pragma unroll
    for (int k = 0; k < QM; ++k) {
        qset(P.ls_lo, k, 0);
        qset(P.ls_hi, k, 0);
        qset(P.bottom, k, 0);
        qset(P.top_cache, k, 0);
        qset(P.pend, k, 0);
    }
    P.cur_q = 0;
}

struct TaskCtxT {
    const Arena* A;
    WarpShared* S;
};

// ---------------------------------------------------------------------------
// task-id allocation
// ---------------------------------------------------------------------------
static __device__ __noinline__ int alloc_id_slow(const Arena& A, WarpShared& S) {
    int b = atomicAdd(&S.bump, 1);
    if (b < A.ids_per_worker) return A.id_base + S.worker * A.ids_per_worker + b;
    // recycled ids before never-used ones, so the arena is only consumed as far
    // as the live set requires (rare: the per-round refill keeps the cache full)
    const Ring& r = A.idpool;
    const unsigned cap = 1u << r.cap_log2;
    for (int attempt = 0; attempt < 64; ++attempt) {
        unsigned h = 0;
        if (pool_claim(r, 1u, h) == 1u) {
            for (int spin = 0; spin < (1 << 20); ++spin) {
                unsigned long long w = ld_acquire(&r.slots[h & (cap - 1)]);
                if (ring_word_ready(w, h, r.cap_log2)) return ring_word_value(w);
                __nanosleep(64);
            }
            GTAP_ERROR(A, ERR_TIMEOUT, -1, -1, (int)h, 0);
            return A.total_ids;
        }
        const unsigned t = ld_relaxed(r.tail), hh = ld_relaxed(r.head);
        if (t == hh || t - hh > cap) break;   // pool empty: every id is live
        __nanosleep(32);
    }
    unsigned f = atom_add_relaxed(A.fresh_next, 1u);
    if (f < (unsigned)A.total_ids) return (int)f;
    GTAP_ERROR(A, ERR_POOL_EXHAUSTED, -1, -1, A.total_ids, A.total_ids);
    return A.total_ids;   // the spare record: written to, never staged or run
}

// The lanes of `m` (calling together) add one each to *p with a single
// shared-memory atomic; returns this lane's old value.
__device__ __forceinline__ int warp_agg_inc(int* p, unsigned m) {
    const unsigned lane = lane_id();
    const int leader = __ffs(m) - 1;
    int base = 0;
    if ((int)lane == leader) base = atomicAdd(p, __popc(m));
    base = __shfl_sync(m, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ int alloc_id(const Arena& A, WarpShared& S) {
    const int a = warp_agg_inc(&S.alloc_pos, __activemask());
    if (a < S.avail_n) return S.avail[(S.avail_head + a) & (kAvailCap - 1)];
    return alloc_id_slow(A, S);
}

// Warp-cooperative, after a round: drop the ids the round took from the
// front of the cache ring, append the ids it freed, return surplus ids to the
// global ring and refill from the private range / ring / fresh ids.
static __device__ void id_cache_maintain(const Arena& A, WarpShared& S) {
    const unsigned lane = lane_id();
    __syncwarp();
    const int consumed = min(S.alloc_pos, S.avail_n);
    const int head = (S.avail_head + consumed) & (kAvailCap - 1);
    int n = S.avail_n - consumed;   // cached ids, avail[head], avail[head + 1], ...
    const int nfreed = min(S.freed_n, kFreedCap);
    const int used_this_round = S.alloc_pos;
    int* const ring = S.avail;
    auto at = [&](int i) -> int& { return ring[(head + i) & (kAvailCap - 1)]; };
    // append freed ids; whatever does not fit goes to the global ring
    for (int base = 0; base < nfreed; base += 32) {
        int i = base + (int)lane;
        int id = (i < nfreed) ? S.freed[i] : -1;
        int take = min(32, nfreed - base);
        int room = kAvailCap - n;
        if (take <= room) {
            if ((int)lane < take) at(n + (int)lane) = id;
            n += take;
        } else {
            // push this chunk of freed ids to the recycled-id ring
            ring_push_warp(A, A.idpool, id, take);
        }
        __syncwarp();
    }
    // surplus: give the 32 newest back
    if (n > min(kAvailHigh, A.avail_target + 32)) {
        int id = at(n - 32 + (int)lane);
        __syncwarp();
        ring_push_warp(A, A.idpool, id, 32);
        n -= 32;
    }
    // refill to about twice the last round's demand
    const int target = min(A.avail_target, max(64, 2 * used_this_round));
    for (int chunk = 0; chunk < 6 && n < target; ++chunk) {
        int got = 0;
        // private range first (no memory traffic)
        int b = S.bump;
        if (b < A.ids_per_worker) {
            int k = min(32, A.ids_per_worker - b);
            if ((int)lane < k) at(n + (int)lane) = A.id_base + S.worker * A.ids_per_worker + b + lane;
            got = k;
            __syncwarp();
            if (lane == 0) S.bump = b + k;
        }
        if (got == 0) {
            int id = -1;
            got = ring_pop_warp(A, A.idpool, 32, &id, true);
            if ((int)lane < got) at(n + (int)lane) = id;
        }
        if (got == 0) {
            unsigned f = 0;
            if (lane == 0) f = atom_add_relaxed(A.fresh_next, 32u);
            f = __shfl_sync(0xffffffffu, f, 0);
            if (f < (unsigned)A.total_ids) {
                int k = min(32, A.total_ids - (int)f);
                if ((int)lane < k) at(n + (int)lane) = (int)f + lane;
                got = k;
            }
        }
        n += got;
        if (got == 0) break;
        __syncwarp();
    }
    __syncwarp();
    if (lane == 0) {
        S.avail_head = head;
        S.avail_n = n;
        S.alloc_pos = 0;
        S.freed_n = 0;
        S.alloc_last = used_this_round;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// task ABI used by task bodies (one lane = one task)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int rt_state(const WarpShared& S) { return (int)(S.l_w0[lane_id()] & 0xFFFFu); }

// A detached child that did not fit the staging buffer, once its frame is
// written: the fence orders its record, frame and function pointer before the
// id appears in the overflow queue.
__device__ __forceinline__ void push_overflow_child(const Arena& A, WarpShared& S, int id) {
    fence_acq_rel();
    ring_push_one(A.overflow, id);
#ifndef GTAP_PHASE_TIMERS
    atomicAdd(&S.st[GTAP_STAT_OVERFLOW_PUSHES], 1ull);
#endif
    (void)S;
}

// Allocate a child, write its header, stage it for this round's push.
// Children are invisible to other workers until the task that spawned them
// has filled their frames (reference contract of __gtap_spawn_task: the
// caller writes the frame after this returns).
__device__ __forceinline__ void* rt_spawn(const Arena& A, WarpShared& S, int kind, int q, int* child_count,
                                          int* out_tid, bool retain, bool detached) {
    const unsigned lane = lane_id();
    if ((unsigned)q >= (unsigned)A.num_queues) {
        GTAP_ERROR(A, ERR_INVALID_QUEUE_IDX, S.l_tid[lane], q, q, A.num_queues);
        q = 0;
    }
    int id = alloc_id(A, S);
    if (out_tid) *out_tid = id;
    if (id >= A.total_ids) return frame_of(A, A.total_ids);   // allocation failed; error already recorded
#ifdef GTAP_DEBUG_IDS
    if (atomicExch(&A.dbg_live[id], 1) != 0) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, id, q, 1, S.l_tid[lane]);
    atomicExch(&A.dbg_exec[id], 0);
#endif
    TaskHeader* h = hdr_of(A, id);
    int4 hw;
    hw.x = (int)((unsigned)kind << 16 | (unsigned)(q | (retain ? kFlagRetain : 0)) << 24);
    hw.y = detached ? -1 : S.l_tid[lane];
    hw.z = 0;
    hw.w = S.l_root[lane];
    *reinterpret_cast<int4*>(h) = hw;
    const unsigned m = __activemask();
    const int s = warp_agg_inc(&S.cnt[q], A.num_queues == 1 ? m : __match_any_sync(m, q));
    bool charged = false;
    if (s < A.spawn_cap) {
        S.sbuf[q * A.spawn_cap + s] = id | (int)(lane << kIdBits);
    } else if (detached) {
        // staging area full: a child that never notifies its parent goes to
        // the global overflow queue instead.  Its creation is charged to its
        // root at once (the round's own charge covers staged children only),
        // and it is pushed when its frame is complete: at this lane's next
        // spawn or when its task returns.  One child per lane waits, so any
        // number of children fits.
        atomicSub(&S.cnt[q], 1);
        const int r = S.l_root[lane];
        red_add_relaxed(&A.outstanding[r], 1ll);
        red_add_relaxed(reinterpret_cast<long long*>(&A.results[r].tasks), 1ll);
        atomicAdd(&S.st[GTAP_STAT_TASKS], 1ull);
        charged = true;
        const int prev = S.l_pend[lane];
        S.l_pend[lane] = id;
        if (prev >= 0) push_overflow_child(A, S, prev);
    } else {
        GTAP_ERROR(A, ERR_SPAWN_BUFFER_OVERFLOW, S.l_tid[lane], q, s, A.spawn_cap);
    }
    if (child_count) ++*child_count;
    if (!detached) S.l_spawned[lane] += 1;
    if (!charged) S.l_created[lane] += 1;
    return frame_of(A, id);
}

// The lanes of `m` (calling together) claim two entries each of the counter
// *p with one shared-memory atomic, laid out as two calls of warp_agg_inc
// would lay them out: the first entries of all lanes, then the second ones.
// Returns this lane's first entry; its second is that + popc(m).
__device__ __forceinline__ int warp_agg_inc2(int* p, unsigned m) {
    const unsigned lane = lane_id();
    const int leader = __ffs(m) - 1;
    int base = 0;
    if ((int)lane == leader) base = atomicAdd(p, 2 * __popc(m));
    base = __shfl_sync(m, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

// Two attached children on queue 0 at once (the built-in fib): one claim on
// the id cache and one on the staging buffer serve both, instead of one each
// per child.  Same effect as two rt_spawn(kind, 0, ...) calls by the lanes
// of the call: the same ids and staging entries, both headers written, both
// children counted for the lane.  When an id cannot be had (the arena is exhausted, an error is
// recorded), the lanes of the call stage their children one by one.
__device__ __forceinline__ void rt_spawn_pair(const Arena& A, WarpShared& S, int kind, int* child_count,
                                              void** frame1, void** frame2) {
    const unsigned lane = lane_id();
    const unsigned m = __activemask();
    const int nm = __popc(m);
    const int a = warp_agg_inc2(&S.alloc_pos, m);
    const int id1 = a < S.avail_n ? S.avail[(S.avail_head + a) & (kAvailCap - 1)] : alloc_id_slow(A, S);
    const int id2 = a + nm < S.avail_n ? S.avail[(S.avail_head + a + nm) & (kAvailCap - 1)] : alloc_id_slow(A, S);
    const int4 hw = make_int4((int)((unsigned)kind << 16), S.l_tid[lane], 0, S.l_root[lane]);
    const bool ok1 = id1 < A.total_ids, ok2 = id2 < A.total_ids;
#ifdef GTAP_DEBUG_IDS
    if (ok1 && atomicExch(&A.dbg_live[id1], 1) != 0) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, id1, 0, 1, S.l_tid[lane]);
    if (ok1) atomicExch(&A.dbg_exec[id1], 0);
    if (ok2 && atomicExch(&A.dbg_live[id2], 1) != 0) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, id2, 0, 1, S.l_tid[lane]);
    if (ok2) atomicExch(&A.dbg_exec[id2], 0);
#endif
    if (ok1) *reinterpret_cast<int4*>(hdr_of(A, id1)) = hw;
    if (ok2) *reinterpret_cast<int4*>(hdr_of(A, id2)) = hw;
    const int tag = (int)(lane << kIdBits);
    if (__all_sync(m, ok1 && ok2)) {
        const int s = warp_agg_inc2(&S.cnt[0], m);
        if (s < A.spawn_cap) S.sbuf[s] = id1 | tag;
        if (s + nm < A.spawn_cap) S.sbuf[s + nm] = id2 | tag;
        if (s + nm >= A.spawn_cap) GTAP_ERROR(A, ERR_SPAWN_BUFFER_OVERFLOW, S.l_tid[lane], 0, s + nm, A.spawn_cap);
        S.l_created[lane] += 2;
    } else {
        // a failed allocation takes no staging entry (as in rt_spawn)
        int made = 0;
        const unsigned m1 = __ballot_sync(m, ok1);
        if (ok1) {
            const int s = warp_agg_inc(&S.cnt[0], m1);
            if (s < A.spawn_cap) S.sbuf[s] = id1 | tag;
            else GTAP_ERROR(A, ERR_SPAWN_BUFFER_OVERFLOW, S.l_tid[lane], 0, s, A.spawn_cap);
            ++made;
        }
        const unsigned m2 = __ballot_sync(m, ok2);
        if (ok2) {
            const int s = warp_agg_inc(&S.cnt[0], m2);
            if (s < A.spawn_cap) S.sbuf[s] = id2 | tag;
            else GTAP_ERROR(A, ERR_SPAWN_BUFFER_OVERFLOW, S.l_tid[lane], 0, s, A.spawn_cap);
            ++made;
        }
        S.l_created[lane] += made;
    }
    if (child_count) *child_count += 2;
    S.l_spawned[lane] += 2;
    *frame1 = frame_of(A, ok1 ? id1 : A.total_ids);
    *frame2 = frame_of(A, ok2 ? id2 : A.total_ids);
}

// taskwait: returns true if the task must suspend (children outstanding).
// then_sum: the task's code after this taskwait is the kJoinSumBit
// continuation, which the child completing the join runs in place.
__device__ __forceinline__ bool rt_join(const Arena& A, WarpShared& S, int child_count, int next_state, int q_after,
                                        bool then_sum = false) {
    const unsigned lane = lane_id();
    if ((unsigned)q_after >= (unsigned)A.num_queues) {
        GTAP_ERROR(A, ERR_INVALID_QUEUE_IDX_AFTER_JOIN, S.l_tid[lane], q_after, q_after, A.num_queues);
        q_after = 0;
    }
    S.l_spawned[lane] = 0;
    if (child_count == 0) {
        S.l_w0[lane] = (S.l_w0[lane] & 0xFFFF0000u) | (unsigned)(next_state & 0xFFFF);
        return false;
    }
    unsigned w0 = (S.l_w0[lane] & 0xFFFF0000u) | (unsigned)(next_state & 0xFFFF);
    S.l_w0[lane] = w0;
    int4 hw;
    hw.x = (int)w0;
    hw.y = S.l_parent[lane];
    hw.z = (child_count & kJoinCountMask) | (q_after << 24) | (then_sum ? kJoinSumBit : 0);
    hw.w = S.l_root[lane];
    *reinterpret_cast<int4*>(hdr_of(A, S.l_tid[lane])) = hw;
    return true;
}

// Task returned.  Parent notification and id release happen at round end.
__device__ __forceinline__ void rt_finish(const WarpShared& S_, bool retain_override = false) {
    WarpShared& S = const_cast<WarpShared&>(S_);
    const unsigned lane = lane_id();
    const unsigned flags = S.l_w0[lane] >> 24;
    S.l_flags[lane] |= kLaneFinished | (((flags & kFlagRetain) || retain_override) ? kLaneRetain : 0);
}

__device__ __forceinline__ void rt_release_id_dbg(const Arena& A, int tid) {
#ifdef GTAP_DEBUG_IDS
    if (atomicExch(&A.dbg_live[tid], 0) != 1) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, tid, -1, 2, 0);
#else
    (void)A;
    (void)tid;
#endif
}

// The id returns to this warp's free-id stack at round end; beyond kFreedCap
// releases in one round it goes to the recycled-id ring at once, after a fence
// that completes this lane's earlier accesses to the id's record (the next
// owner rewrites it).
__device__ __forceinline__ void rt_release_id(const Arena& A, WarpShared& S, int tid) {
    const int f = warp_agg_inc(&S.freed_n, __activemask());
    if (f < kFreedCap) {
        S.freed[f] = tid;
    } else {
        fence_acq_rel();
        ring_push_one(A.idpool, tid);
    }
}

// One lane, after its join decrement brought task p's count to zero and
// carried kJoinSumBit: p's continuation runs here instead of in a later round.
// The acquiring decrement made the siblings' results in p's frame visible; the
// sum goes into the grandparent's frame (or the root's result) and p finishes
// (its id goes back, `finished` counts it for the root, which every task of the
// chain shares).  The grandparent's join decrement releases the store; when it
// completes that join too, the walk continues upwards.  Returns the task to
// resume (a completed join without the bit, with its queue in rq), or -1.
// Each step goes to a strict ancestor, so the walk ends within the tree's depth.
static __device__ __noinline__ int join_sum_walk(const Arena& A, WarpShared& S, int p, int& finished, int& rq) {
    for (;;) {
        const int4 h = ld_cg_v4(hdr_of(A, p));
        const int4 f = ld_cg_v4(frame_of(A, p));
        const int gp = h.y;
        const int v = (int)((unsigned)f.y + (unsigned)f.z);
        if (gp >= 0) *reinterpret_cast<int*>(reinterpret_cast<char*>(frame_of(A, gp)) + (f.w & 0xFF)) = v;
        else A.results[h.w].value = v;
        rt_release_id_dbg(A, p);
        if (!(((unsigned)h.x >> 24) & kFlagRetain)) rt_release_id(A, S, p);
        ++finished;
        if (gp < 0) return -1;
        const int old = atom_add_acq_rel(&hdr_of(A, gp)->join, -1);
        if ((old & kJoinCountMask) != 1) return -1;
        if (!(old & kJoinSumBit)) {
            rq = (old >> 24) & 7;
            if (rq >= A.num_queues) rq = 0;
            return gp;
        }
        p = gp;
    }
}

// ---------------------------------------------------------------------------
// root accounting
// ---------------------------------------------------------------------------
static __device__ void complete_root(const Arena& A, int r) {
    gtap_root_result* res = &A.results[r];
    res->t_done_ns = global_ns();
    __threadfence();
    st_release(&res->status, GTAP_ROOT_DONE);
    unsigned c = atomicAdd(A.completed, 1u) + 1u;
    if (A.mode == 2 /* serve */) {
        if (A.done_ring) {
            unsigned slot = (c - 1u) % A.done_ring_cap;
            unsigned long long w = ((unsigned long long)(c - 1u) << 32) | (unsigned)(r + 1);
            volatile unsigned long long* p = A.done_ring + slot;
            *p = w;
            __threadfence_system();
        }
    } else if (c >= (unsigned)A.n_roots) {
        st_release(A.done_flag, 1);
    }
}

// counter update; completes the root when it reaches zero
__device__ __forceinline__ void outstanding_add(const Arena& A, int r, long long d) {
    long long old = atom_add_acq_rel(&A.outstanding[r], d);
    if (old + d == 0) complete_root(A, r);
}

static __device__ void flush_bal(const Arena& A, RootBal& e) {
    if (e.created) red_add_relaxed(reinterpret_cast<long long*>(&A.results[e.root].tasks), (long long)e.created);
    e.created = 0;
    if (e.bal != 0) outstanding_add(A, e.root, -(long long)e.bal);
    e.bal = 0;
}

// lane 0 only
static __device__ void flush_all_bal(const Arena& A, WarpShared& S) {
    for (int i = 0; i < S.nbal; ++i) flush_bal(A, S.bal[i]);
    S.nbal = 0;
}

// Called by one leader lane per distinct root, serialised across leaders.
static __device__ void account_root(const Arena& A, WarpShared& S, int r, int created, int finished) {
    int idx = -1;
    for (int i = 0; i < S.nbal; ++i)
        if (S.bal[i].root == r) { idx = i; break; }
    if (idx < 0 && S.nbal < kRootBalCap) {
        idx = S.nbal++;
        S.bal[idx].root = r;
        S.bal[idx].bal = 0;
        S.bal[idx].created = 0;
    }
    if (idx < 0) {
        // no cache slot: apply directly (creations before publication keep it safe)
        if (created) red_add_relaxed(reinterpret_cast<long long*>(&A.results[r].tasks), (long long)created);
        if (created != finished) outstanding_add(A, r, (long long)(created - finished));
        return;
    }
    RootBal& e = S.bal[idx];
    e.touched = 1;
    e.created += created;
    e.bal += finished - created;
    if (e.bal < 0) {
        int top = kBalChunk - e.bal;
        outstanding_add(A, r, (long long)top);
        e.bal = kBalChunk;
    }
}

// lane 0: flush entries not touched this round so completions are seen promptly
static __device__ void age_bal(const Arena& A, WarpShared& S) {
    int j = 0;
    for (int i = 0; i < S.nbal; ++i) {
        if (S.bal[i].touched) {
            S.bal[i].touched = 0;
            if (j != i) S.bal[j] = S.bal[i];
            ++j;
        } else {
            flush_bal(A, S.bal[i]);
        }
    }
    S.nbal = j;
}

// ---------------------------------------------------------------------------
// deque operations
// ---------------------------------------------------------------------------
// Owner pop: LIFO, up to 32 newest published tasks of queue k.
template <int QM>
static __device__ int pop_own(const Arena& A, WarpShared& S, QueuePos<QM>& P, int k, int& my_tid) {
    const unsigned lane = lane_id();
    if (((qget(P.bottom, k) - qget(P.top_cache, k)) & kPosMask) == 0) return 0;  // top only grows: surely empty
    int got = 0;
    unsigned b = 0, top = qget(P.top_cache, k);
    if (lane == 0) {
        unsigned long long* c = dq_ctl_ptr(A, k, S.worker);
        unsigned long long wv = ld_relaxed(c);
        for (int i = 0; i < 16; ++i) {
            unsigned sz = dq_size(wv);
            top = dq_top(wv);
            if (sz == 0) break;
            unsigned take = sz < 32u ? sz : 32u;
            unsigned long long old = atom_cas_acquire(c, wv, dq_owner_pop(wv, take));
            if (old == wv) {
                got = (int)take;
                b = dq_bottom(wv);
#ifdef GTAP_QUEUE_CHECKS
                if (take > sz || sz > (1u << A.deque_cap_log2)) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, (int)take, k, 23, (int)sz);
#endif
#ifdef GTAP_DEBUG_IDS
                if (b != qget(P.bottom, k)) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, (int)b, k, 11, (int)qget(P.bottom, k));
#endif
                break;
            }
            wv = old;
        }
        if (got) S.st[GTAP_STAT_POPS] += 1;
    }
    got = __shfl_sync(0xffffffffu, got, 0);
    b = __shfl_sync(0xffffffffu, b, 0);
    qset(P.top_cache, k, __shfl_sync(0xffffffffu, top, 0));
    if (got) qset(P.bottom, k, (b - (unsigned)got) & kPosMask);
    if ((int)lane < got) {
        my_tid = ld_relaxed(dq_slot_ptr(A, k, S.worker, b - (unsigned)got + lane));
#ifdef GTAP_DEBUG_IDS
        const unsigned pos = (b - (unsigned)got + lane) & kPosMask;
        const size_t si = dq_slot_ptr(A, k, S.worker, pos) - A.dq_slots;
        if (ld_cg((const int*)&A.dbg_slotpos[si]) != (int)pos)
            GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, my_tid, k, 12, (int)pos);
#endif
    }
    return got;
}

__device__ __forceinline__ unsigned xorshift32(unsigned& s) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return s;
}

// Thief: probe up to probe_width random victims in parallel (one lane each),
// take up to steal_batch (at most half) of the fullest one's queue k with one
// CAS on its control word.
static __device__ int steal(const Arena& A, WarpShared& S, int k, unsigned& rng, int& last_victim, int& my_tid) {
    const unsigned lane = lane_id();
    const int W = A.num_workers;
    if (W < 2) return 0;
    int victim = -1;
    unsigned long long wv = 0;
    unsigned sz = 0;
    if ((int)lane < A.probe_width) {
        int v;
        if (lane == 0 && A.victim_policy == GTAP_VICTIM_LAST_SUCCESS && last_victim >= 0) {
            v = last_victim;
        } else {
            v = (int)(xorshift32(rng) % (unsigned)(W - 1));
            if (v >= S.worker) ++v;
        }
        victim = v;
        wv = ld_acquire(dq_ctl_ptr(A, k, v));
        sz = dq_size(wv);
    }
    // argmax over lanes (largest size, lowest lane on ties)
    unsigned key = (sz << 5) | (31u - lane);
    if (sz > (1u << 21)) key = 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if (lane == 0) S.st[GTAP_STAT_STEAL_ATTEMPTS] += 1;
    if ((key >> 5) == 0) return 0;
    int src = 31 - (int)(key & 31u);
    victim = __shfl_sync(0xffffffffu, victim, src);
    wv = __shfl_sync(0xffffffffu, wv, src);
    __syncwarp();   // orders the probing lane's acquire before every lane's slot reads
    unsigned long long* c = dq_ctl_ptr(A, k, victim);
    for (int attempt = 0; attempt < 3; ++attempt) {
        unsigned size = dq_size(wv);
        if (size == 0 || size > (1u << 20)) return 0;
        unsigned t = dq_top(wv);
        unsigned half = (size + 1u) >> 1;
        unsigned n = half < (unsigned)A.steal_batch ? half : (unsigned)A.steal_batch;
        int id = -1;
#ifdef GTAP_DEBUG_IDS
        int shadow_ok = 1;
#endif
        if (lane < n) {
            // Acquire: the read must be complete before lane 0's CAS claims the
            // batch.  Once the CAS lands the owner may refill this slot for the
            // next lap, and a relaxed load still in flight could return that
            // newer value (a barrier alone does not wait for pending loads).
            id = ld_acquire(dq_slot_ptr(A, k, victim, t + lane));
#ifdef GTAP_DEBUG_IDS
            const unsigned pos = (t + lane) & kPosMask;
            const size_t si = dq_slot_ptr(A, k, victim, pos) - A.dq_slots;
            shadow_ok = ld_cg((const int*)&A.dbg_slotpos[si]) == (int)pos;
#endif
        }
        __syncwarp();
        unsigned long long old = 0;
        if (lane == 0) old = atom_cas_acquire(c, wv, dq_with_top(wv, t + n));
        old = __shfl_sync(0xffffffffu, old, 0);
        if (old == wv) {
#ifdef GTAP_DEBUG_IDS
            if (lane < n && !shadow_ok) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, id, k, 13, (int)((t + lane) & kPosMask));
#endif
#ifdef GTAP_QUEUE_CHECKS
            if (lane == 0 && (n > size || size > (1u << A.deque_cap_log2)))
                GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, (int)n, k, 22, (int)size);
#endif
            if (lane < n) my_tid = id;
            if (lane == 0) {
                S.st[GTAP_STAT_STEAL_SUCCESSES] += 1;
                S.st[GTAP_STAT_STOLEN_TASKS] += n;
            }
            last_victim = victim;
            return (int)n;
        }
        wv = old;
    }
    return 0;
}

// Write m entries src[(start + i) & mask] into this warp's deque of queue k
// (the owner's bottom moves at once; thieves see them only after
// publish_commit), spilling to the overflow queue when the deque is full.
template <int QM>
static __device__ void publish_stage(const Arena& A, WarpShared& S, QueuePos<QM>& P, int k, const int* base,
                                     unsigned start, unsigned mask, int m) {
    const unsigned lane = lane_id();
    const unsigned cap = 1u << A.deque_cap_log2;
    auto src = [&](int i) { return base[(start + (unsigned)i) & mask]; };
    unsigned used = (qget(P.bottom, k) - qget(P.top_cache, k)) & kPosMask;
    if (used + (unsigned)m > cap) {
        unsigned long long wv = 0;
        if (lane == 0) wv = ld_relaxed(dq_ctl_ptr(A, k, S.worker));
        wv = __shfl_sync(0xffffffffu, wv, 0);
        qset(P.top_cache, k, dq_top(wv));
        used = (qget(P.bottom, k) - qget(P.top_cache, k)) & kPosMask;
    }
    int direct = m;
    if (used + (unsigned)m > cap) direct = (int)(cap - used);
#ifdef GTAP_QUEUE_CHECKS
    if (lane == 0 && used > cap) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, (int)used, k, 20, (int)cap);
#endif
    if (direct > 0) {
        const unsigned b = qget(P.bottom, k);
#ifdef GTAP_QUEUE_CHECKS
        if (lane == 0) {
            unsigned long long w = ld_relaxed(dq_ctl_ptr(A, k, S.worker));
            if (((dq_bottom(w) + (unsigned)qget(P.pend, k)) & kPosMask) != b)
                GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, (int)dq_bottom(w), k, 21, (int)b);
            if (((b - dq_top(w)) & kPosMask) + (unsigned)direct > cap)
                GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, (int)dq_top(w), k, 24, (int)qget(P.top_cache, k));
        }
#endif
        for (int e = (int)lane; e < direct; e += 32) {
            *dq_slot_ptr(A, k, S.worker, b + (unsigned)e) = src(e) & kIdMask;
#ifdef GTAP_DEBUG_IDS
            if (ld_cg(&A.dbg_live[src(e) & kIdMask]) != 1) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, src(e) & kIdMask, k, 14, e);
            const unsigned pos = (b + (unsigned)e) & kPosMask;
            A.dbg_slotpos[dq_slot_ptr(A, k, S.worker, pos) - A.dq_slots] = pos;
#endif
        }
        qset(P.bottom, k, (b + (unsigned)direct) & kPosMask);
        qset(P.pend, k, qget(P.pend, k) + (direct));
    }
    // the rest spills to the global overflow queue (its own fence: rare)
    for (int base_i = direct; base_i < m; base_i += 32) {
        int take = min(32, m - base_i);
        int id = ((int)lane < take) ? (src(base_i + (int)lane) & kIdMask) : 0;
#ifdef GTAP_DEBUG_IDS
        if ((int)lane < take && ld_cg(&A.dbg_live[id]) != 1) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, id, k, 16, base_i);
#endif
        fence_acq_rel();
        ring_push_warp(A, A.overflow, id, take);
#ifndef GTAP_PHASE_TIMERS
        if (lane == 0) S.st[GTAP_STAT_OVERFLOW_PUSHES] += (unsigned long long)take;
#endif
    }
    __syncwarp();   // the source entries are read before any lane overwrites them
}

// One warp-wide fence orders every store this warp made so far (task
// records, results, deque slots) before what follows; then lane 0 moves the
// bottoms of the deques publish_stage wrote, making those entries stealable.
// fence: also when nothing is pending.
template <int QM>
static __device__ void publish_commit(const Arena& A, WarpShared& S, QueuePos<QM>& P, bool fence) {
    const unsigned lane = lane_id();
    bool any = false;
#pragma unroll
    for (int k = 0; k < QM; ++k) any |= P.pend[k] != 0;
    if (!any && !fence) return;
    fence_acq_rel();
    __syncwarp();   // every lane's fence is done before lane 0 publishes
    if (any) {
        if (lane == 0) {
            for (int k = 0; k < queue_count<QM>(A); ++k) {
                const int d = qget(P.pend, k);
                if (d) {
                    red_add_relaxed(dq_ctl_ptr(A, k, S.worker), (unsigned long long)d << kPosBits);
#ifndef GTAP_PHASE_TIMERS
                    S.st[GTAP_STAT_PUBLISHED] += (unsigned long long)d;
#endif
                }
            }
        }
#pragma unroll
        for (int k = 0; k < QM; ++k) P.pend[k] = 0;
    }
}

// Stage and publish at once.
template <int QM>
static __device__ void publish_src(const Arena& A, WarpShared& S, QueuePos<QM>& P, int k, const int* base, unsigned start,
                                   unsigned mask, int m) {
    publish_stage(A, S, P, k, base, start, mask, m);
    publish_commit(A, S, P, false);
}

// ---------------------------------------------------------------------------
// profiling (reference gtap_profile_thread.cuh timelines)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void prof_having(const Arena& A, WarpShared& S) {
    if (A.prof_cap > 0 && lane_id() == 0 && S.prof_h < A.prof_cap) {
        A.prof_having[(size_t)S.worker * A.prof_cap + S.prof_h] = (long long)global_ns();
        S.prof_h++;
    }
}
__device__ __forceinline__ void prof_working(const Arena& A, WarpShared& S, int nb) {
    if (A.prof_cap > 0 && lane_id() == 0 && S.prof_w < A.prof_cap) {
        size_t i = (size_t)S.worker * A.prof_cap + S.prof_w;
        A.prof_working[i] = (long long)global_ns();
        A.prof_tasks[i] = nb;
        S.prof_w++;
    }
}

// ---------------------------------------------------------------------------
// admission: claim roots from the root table (batch) or the published ring (serve)
// ---------------------------------------------------------------------------
template <class Prog>
static __device__ int admit(const Arena& A, WarpShared& S, int& my_tid) {
    const unsigned lane = lane_id();
    int first = 0, k = 0;
    if (lane == 0) {
        unsigned limit;
        limit = (A.mode == 2) ? ld_acquire(A.published) : (unsigned)A.n_roots;
        // admission by free task-frame memory: never-used + recycled ids
        unsigned fresh = ld_relaxed(A.fresh_next);
        unsigned pool = ld_relaxed(A.idpool.tail) - ld_relaxed(A.idpool.head);
        long long free_ids = (long long)A.total_ids - (long long)fresh + (long long)pool;
        if (free_ids < (long long)A.admit_watermark) limit = 0;
        if (A.max_inflight > 0) {
            // admitted - completed < max_inflight
            const unsigned done = ld_relaxed(A.completed);
            const unsigned cap = done + (unsigned)A.max_inflight;
            if (cap < limit) limit = cap;
        }
        for (int attempt = 0; attempt < 8; ++attempt) {
            unsigned c = ld_relaxed(A.next_root);
            if (c >= limit) break;
            unsigned take = limit - c;
            if (take > (unsigned)A.admit_batch) take = (unsigned)A.admit_batch;
            if (atom_cas_relaxed(A.next_root, c, c + take) == c) {
                first = (int)c;
                k = (int)take;
                break;
            }
        }
    }
    k = __shfl_sync(0xffffffffu, k, 0);
    first = __shfl_sync(0xffffffffu, first, 0);
    if (k == 0) return 0;
    if ((int)lane < k) {
        int idx = first + (int)lane;
        int slot = (A.mode == 2) ? (int)((unsigned)idx % (unsigned)A.n_roots) : idx;
        const gtap_root& rd = A.roots[slot];
        int id = alloc_id(A, S);
        if (id >= A.total_ids) id = A.total_ids;   // error recorded; the launch aborts
#ifdef GTAP_DEBUG_IDS
        if (id < A.total_ids) {
            if (atomicExch(&A.dbg_live[id], 1) != 0) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, id, -1, 4, 0);
            atomicExch(&A.dbg_exec[id], 0);
        }
#endif
        int kind = Prog::root_kind(rd.kind);
        bool valid = true;
        if (kind < 0) {
            GTAP_ERROR(A, ERR_INVALID_KIND, id, -1, rd.kind, GTAP_KIND_COUNT);
            kind = 0;
            valid = false;
        } else if (!Prog::root_args_ok(rd)) {
            GTAP_ERROR(A, ERR_INVALID_ARGUMENT, id, -1, rd.kind, 0);
            kind = 0;
            valid = false;
        }
        TaskHeader* h = hdr_of(A, id);
        int4 hw;
        hw.x = (int)((unsigned)kind << 16);
        hw.y = -1;
        hw.z = 0;
        hw.w = slot;
        *reinterpret_cast<int4*>(h) = hw;
        if (valid) Prog::init_root(A, rd, frame_of(A, id));
        gtap_root_result* res = &A.results[slot];
        // a serve-mode slot is reused after its previous root was polled:
        // everything the root accumulates starts here
        res->value = 0;
        res->tasks = 1;   // the root itself; its descendants are added as they are created
        res->t_done_ns = 0;
        res->t_admit_ns = global_ns();
        res->index = idx;
        res->status = GTAP_ROOT_RUNNING;
        // the root counts as one outstanding task from here on; its finish
        // enters this or another warp's balance like any other task
        atom_add_acq_rel(&A.outstanding[slot], 1ll);
        S.l_created[lane] = 0;
        S.l_root[lane] = slot;
        my_tid = id;
    }
    __syncwarp();
    if (lane == 0) S.st[GTAP_STAT_TASKS] += (unsigned long long)k;
    return k;
}

// ---------------------------------------------------------------------------
// the persistent worker loop
// ---------------------------------------------------------------------------
template <class Prog, int QM>
static __device__ void worker_loop(const Arena& A, WarpShared& S, int initial_tid) {
    const unsigned lane = lane_id();
    QueuePos<QM> P;
    queue_pos_init(P);
    int my_tid = (initial_tid >= 0 && lane == 0) ? initial_tid : -1;
    int nb = initial_tid >= 0 ? 1 : 0;
    unsigned rng = 0x9E3779B9u ^ (unsigned)(S.worker * 2654435761u) ^ (lane * 0x85EBCA6Bu) ^ (unsigned)clock64();
    if (rng == 0) rng = 1;
    int last_victim = -1;
    int backoff = 0;
    bool having = false;
    // watchdog (lane 0): a batch launch is bounded as a whole; a serve
    // session only while roots are outstanding and none completes
    if (lane == 0) {
        S.t_watch = global_ns();
        S.seen_done = 0;
    }
    auto watchdog_expired = [&]() -> bool {
        const unsigned long long now = global_ns();
        if (A.mode == 2) {
            const unsigned c = ld_relaxed(A.completed);
            if (c != S.seen_done || c >= ld_relaxed(A.published)) {
                S.seen_done = c;
                S.t_watch = now;
                return false;
            }
        }
        return now - S.t_watch > A.watchdog_ns;
    };
    int round = 0;
    bool staged = false;                     // this round's records are in S.rstage (copies in flight)
    int src_kind = 0;                        // debug builds: where this round's tasks came from
    bool idle = false;                       // counted in the hungry replicas
    unsigned long long idle_since = 0;       // lane 0: start of the current idle stretch
    int* const hungry_mine = A.hungry + (S.worker % kHungryReplicas) * kHungryStride;
    auto hungry_add = [&](int d) {
        for (int r = 0; r < kHungryReplicas; ++r) red_add_relaxed_i32(A.hungry + r * kHungryStride, d);
    };

    for (;;) {
        GTAP_PHASE_MARK(ph0);
        S.l_flags[lane] = 0;
        S.l_created[lane] = 0;
        __syncwarp();

        if (nb == 0) {
            // acquire: own deque, then steal, per EPAQ queue starting at cur_q
            // (reference :896-926), then the overflow queue, then new roots.
            const int Q = queue_count<QM>(A);
            for (int kk = 0; kk < Q && nb == 0; ++kk) {
                int k = (P.cur_q + kk) % Q;
                nb = pop_own(A, S, P, k, my_tid);
                src_kind = 1;
                if (nb == 0) {
                    nb = steal(A, S, k, rng, last_victim, my_tid);
                    src_kind = 2;
                }
                if (nb) {
                    P.cur_q = k;
                }
            }
            if (nb == 0) {
                nb = ring_pop_warp(A, A.overflow, 32, &my_tid);
                src_kind = 3;
            }
            if (nb == 0) {
                nb = admit<Prog>(A, S, my_tid);
                src_kind = 4;
            }
            __syncwarp();
            if (nb == 0) {
                if (having) {
                    prof_having(A, S);
                    having = false;
                }
                int stop = 0;
                if (lane == 0) {
                    if (!idle && A.publish_lazy) hungry_add(1);
                    if (!idle) idle_since = global_ns();
                    flush_all_bal(A, S);
                    S.st[GTAP_STAT_IDLE_POLLS] += 1;
                    if (ld_acquire(A.done_flag) != 0 || aborted(A)) stop = 1;
                    if (A.mode == 2 && ld_relaxed(A.shutdown) != 0) {
                        unsigned pub = ld_acquire(A.published);
                        if (ld_acquire(A.completed) >= pub && ld_relaxed(A.next_root) >= pub) stop = 1;
                    }
                    if (!stop && watchdog_expired()) {
                        GTAP_ERROR(A, ERR_TIMEOUT, -1, -1, 0, 0);
                        stop = 1;
                    }
                }
                idle = true;
                stop = __shfl_sync(0xffffffffu, stop, 0);
                if (stop) {
#ifndef GTAP_PHASE_TIMERS
                    if (lane == 0) S.st[GTAP_STAT_IDLE_NS] += global_ns() - idle_since;
#endif
                    break;
                }
                if (backoff < 6) ++backoff;
                __nanosleep(32u << backoff);
                continue;
            }
            if (idle && lane == 0 && A.publish_lazy) hungry_add(-1);
#ifndef GTAP_PHASE_TIMERS
            if (idle && lane == 0) S.st[GTAP_STAT_IDLE_NS] += global_ns() - idle_since;
#endif
            idle = false;
            backoff = 0;
            if (!having) {
                prof_having(A, S);
                having = true;
            }
        }

        GTAP_PHASE_MARK(ph1);
        GTAP_PHASE_ADD(10, ph0, ph1);
        // ---- execute: lane i runs task my_tid ----
        int hv = 0;
        if (lane == 0 && A.publish_lazy) hv = ld_relaxed(hungry_mine);   // consumed at round end
        prof_working(A, S, nb);
        int4 hw = make_int4(0, -1, 0, 0), fw0 = make_int4(0, 0, 0, 0), fw1 = fw0;
        unsigned long long fn = 0;
        int bad = 0;
        if (staged) rec_stage_wait();
        // Lanes [run_lo, nb) run a task in this pass.  With sub_rounds > 0, a
        // round whose tasks leave lanes idle runs up to sub_rounds more passes
        // on them, each over the newest children the passes before it staged
        // (they would otherwise wait for the next round): a tree's ramp-up
        // and drain go down several levels per round.
        int run_lo = 0;
#ifdef GTAP_PHASE_TIMERS
        long long ph1b = 0;
#endif
        for (int pass = 0;; ++pass) {
        if ((int)lane >= run_lo && (int)lane < nb) {
            if ((unsigned)my_tid >= (unsigned)A.total_ids) {
                bad = 1;
            } else {
                // header, the first 32 frame bytes and (programs that call
                // through a function table) the task function, in one round
                // trip, or from the record stage the previous round filled
                const char* rec = A.records + (size_t)my_tid * A.rec_stride;
                if (staged && pass == 0) {
                    const int4* st4 = S.rstage + lane * 3;
                    hw = st4[0];
                    if (Prog::kFrameWords) {
                        fw0 = st4[1];
                        if (A.rec_stride >= 48) fw1 = st4[2];
                    }
                } else {
                    hw = ld_data_v4(rec);
                    if (Prog::kFrameWords) {
                        fw0 = ld_data_v4(rec + 16);
                        if (A.rec_stride >= 48) fw1 = ld_data_v4(rec + 32);
                    }
                }
                if (Prog::kFuncTable) fn = ld_data_u64(reinterpret_cast<const unsigned long long*>(A.funcs) + my_tid);
                if ((unsigned)hw.w >= (unsigned)A.n_roots || hw.y < -1 || hw.y >= A.total_ids) bad = 2;
            }
            if (bad) GTAP_ERROR(A, ERR_INVALID_ARGUMENT, my_tid, -1, bad == 1 ? my_tid : hw.w, A.total_ids);
        }
        if (__any_sync(0xffffffffu, bad)) break;   // corrupted id or header: leaves the passes, then the loop
#ifdef GTAP_PHASE_TIMERS
        if (pass == 0) {
            GTAP_PHASE_MARK_AFTER(ph1b_, hw.x ^ fw0.x ^ fw1.w ^ (int)fn);
            GTAP_PHASE_ADD(9, ph1, ph1b_);
            ph1b = ph1b_;
        }
#endif
#ifdef GTAP_DEBUG_IDS
        if ((int)lane >= run_lo && (int)lane < nb) {
            if (ld_cg(&A.dbg_live[my_tid]) != 1) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, my_tid, src_kind, 3, (int)lane * 1000 + nb);
            int prev = atomicAdd(&A.dbg_exec[my_tid], 1);
            if ((hw.x & 0xFFFF) == 0 && prev != 0) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, my_tid, -1, 5, prev);
        }
#endif
        if ((int)lane >= run_lo && (int)lane < nb) {
            S.l_tid[lane] = my_tid;
            S.l_w0[lane] = (unsigned)hw.x;
            S.l_parent[lane] = hw.y;
            S.l_root[lane] = hw.w;
            S.l_spawned[lane] = 0;
            S.l_value[lane] = 0;
            Prog::exec(A, S, (int)(((unsigned)hw.x >> 16) & 0xFFu), my_tid, frame_of(A, my_tid), fw0, fw1, fn);
        }
        __syncwarp();
        // another pass: single queue, every staged child in the buffer, and
        // no task of the round returned with children outstanding (those
        // children become orphans at round end, so none may run before it)
        if (!Prog::kSubRounds || pass >= A.sub_rounds || nb >= kWarp) break;
        {
            const int have = S.cnt[0];
            const bool orphans = __any_sync(0xffffffffu, (int)lane < nb && (S.l_flags[lane] & kLaneFinished) &&
                                                             S.l_spawned[lane] > 0);
            if (queue_count<QM>(A) != 1 || have <= 0 || have > A.spawn_cap || orphans) break;
            const int k = min(have, kWarp - nb);
            // lane nb + j takes the j-th newest staged child; the staging
            // entries were written (and the children's records and frames)
            // before the warp barrier above
            if ((int)lane >= nb && (int)lane < nb + k) my_tid = S.sbuf[have - 1 - ((int)lane - nb)] & kIdMask;
            __syncwarp();
            if (lane == 0) S.cnt[0] = have - k;
            __syncwarp();
            run_lo = nb;
            nb += k;
        }
        }
        if (__any_sync(0xffffffffu, bad)) break;   // corrupted id or header: stop this worker, launch aborts
        GTAP_PHASE_MARK(ph2);
        GTAP_PHASE_ADD(11, ph1b, ph2);
        // ---- leaf work the round's tasks left for the whole warp ----
        // (sorted runs and merges; done before any parent learns that the
        // task finished, and fenced so the parent sees the data)
        const int lane_flags = S.l_flags[lane];
        const unsigned leaves = __ballot_sync(0xffffffffu, (int)lane < nb && (lane_flags & kLaneLeaf));
        if (leaves) {
            Prog::warp_leaves(A, S, leaves, (int)(((unsigned)hw.x >> 16) & 0xFFu), fw0, fw1);
            fence_acq_rel();
            __syncwarp();
        }
        prof_working(A, S, nb);

        // ---- round end ----
        int nb_next = 0, next_tid = -1;
        const bool active = (int)lane < nb;
        const unsigned fin = __ballot_sync(0xffffffffu, active && (lane_flags & kLaneFinished));
        const bool my_fin = active && ((fin >> lane) & 1u);
        const unsigned spawners = __ballot_sync(0xffffffffu, active && S.l_spawned[lane] > 0);
        // (0) the children this round created count for their roots before
        //     any of them can be seen by another warp: one that ran and
        //     finished elsewhere before its creation was counted could bring
        //     its root's counter to zero early.  One leader per distinct root.
        const int r0 = S.l_root[0];   // lane 0 always runs a task when nb > 0
        const bool one_root = __all_sync(0xffffffffu, !active || S.l_root[lane] == r0);
        const int my_root = active ? S.l_root[lane] : -1;
        const unsigned grp = one_root ? 0xffffffffu : __match_any_sync(0xffffffffu, my_root);
        {
            const int created = active ? S.l_created[lane] : 0;
            if (__any_sync(0xffffffffu, created != 0)) {
                if (one_root) {
                    const int c_sum = (int)__reduce_add_sync(0xffffffffu, (unsigned)created);
                    if (lane == 0) account_root(A, S, r0, c_sum, 0);
                } else {
                    int c_sum = 0;
                    if (active) c_sum = (int)__reduce_add_sync(grp, (unsigned)created);
                    unsigned leaders = __ballot_sync(0xffffffffu, active && c_sum != 0 && (unsigned)__ffs(grp) - 1u == lane);
                    while (leaders) {
                        if (lane == (unsigned)__ffs(leaders) - 1u) account_root(A, S, my_root, c_sum, 0);
                        __syncwarp();
                        leaders &= leaders - 1u;
                    }
                }
                __syncwarp();
            }
        }
        //     Detached children that did not fit the staging buffer and still
        //     wait (one per lane, charged when spawned): their frames are
        //     complete now that the task bodies returned.
        {
            const int pend = S.l_pend[lane];
            const unsigned pm = __ballot_sync(0xffffffffu, pend >= 0);
            if (pm) {
                S.l_pend[lane] = -1;
                fence_acq_rel();
                __syncwarp();   // every lane's frame stores are ordered before any push
                const int n = __popc(pm);
                const int v = __shfl_sync(0xffffffffu, pend, (int)lane < n ? (int)__fns(pm, 0, (int)lane + 1) : 0);
                ring_push_warp(A, A.overflow, v, n);
#ifndef GTAP_PHASE_TIMERS
                if (lane == 0) S.st[GTAP_STAT_OVERFLOW_PUSHES] += (unsigned long long)n;
#endif
            }
        }
        // (1) orphans: children of tasks that returned without a taskwait
        if (fin & spawners) {
            for (int q = 0; q < queue_count<QM>(A); ++q) {
                const int n = min(S.cnt[q], A.spawn_cap);
                const int* sb = S.sbuf + q * A.spawn_cap;
                for (int e = (int)lane; e < n; e += 32) {
                    unsigned ent = (unsigned)sb[e];
                    unsigned sp = ent >> kIdBits;
                    if ((fin & spawners) >> sp & 1u) hdr_of(A, (int)(ent & kIdMask))->parent = -1;
                }
            }
            __syncwarp();
        }
        // (2) no fence before the joins: each join decrement is an
        //     acquire-release atomic, which releases the results the lane
        //     wrote into its parent's frame and, through this warp barrier,
        //     the stores of the other lanes before it.  Leaf data is fenced
        //     after the leaf work; orphan marks and children's records reach
        //     other warps only through publication, which has its own fence.
        __syncwarp();
        GTAP_PHASE_MARK(ph3);
        GTAP_PHASE_ADD(12, ph2, ph3);
        // (3) joins: the last child re-enqueues its parent on the resume queue;
        //     release the finished task's id unless its parent reads its frame
        //     In a round of at most join_walk tasks, a completed join whose
        //     continuation only sums two results runs that continuation here
        //     (join_sum_walk), up the ancestors whose joins it completes;
        //     `walked` counts the tasks it finished.  Fuller rounds resume
        //     the parent as a task: a walk step costs dependent round trips
        //     that a full round would wait for, while a resumed parent only
        //     takes a lane of the next round.
        int resumed = -1, rq = 0, walked = 0;
        if (my_fin) {
            const int parent = S.l_parent[lane];
            if (parent >= 0) {
                const int old = atom_add_acq_rel(&hdr_of(A, parent)->join, -1);
                if ((old & kJoinCountMask) == 1) {
                    if (Prog::kJoinSum && (old & kJoinSumBit) && nb <= A.join_walk) {
                        resumed = join_sum_walk(A, S, parent, walked, rq);
                    } else {
                        rq = (old >> 24) & 7;
                        if (rq >= queue_count<QM>(A)) rq = 0;
                        resumed = parent;
                    }
                }
            }
            if (!(lane_flags & kLaneRetain)) {
                rt_release_id_dbg(A, my_tid);
                rt_release_id(A, S, my_tid);
            }
        }
        const unsigned rmask = __ballot_sync(0xffffffffu, resumed >= 0);
        GTAP_PHASE_MARK(ph3b);
        GTAP_PHASE_ADD(7, ph3, ph3b);
        // (4) this round's children join their queue's local stack, and the
        //     parents they resumed go on top of them (newest), so continuations
        //     run first; the busiest queue's newest <= 32 run next (reference
        //     push_batch keeps the newest 32 of k_max); the oldest entries are
        //     written to the deque when a stack overflows or some worker is
        //     hungry (always, with eager publication), and published in (5).
        int kn = -1;
        {
            const int Q = queue_count<QM>(A);
            // eager publication behaves as if some worker were always hungry
            const int hungry = A.publish_lazy ? __shfl_sync(0xffffffffu, hv, 0) : 1;
            const int reserve = A.publish_lazy ? kReserve : 0;
            int best = 0;
            for (int k = 0; k < Q; ++k) {
                const int c = S.cnt[k] + (rmask ? __popc(__ballot_sync(0xffffffffu, resumed >= 0 && rq == k)) : 0);
                if (c > best) {
                    best = c;
                    kn = k;
                }
            }
            for (int k = 0; k < Q; ++k) {
                const int n = min(S.cnt[k], A.spawn_cap);
                const unsigned mk = rmask ? __ballot_sync(0xffffffffu, resumed >= 0 && rq == k) : 0u;
                const int add = __popc(mk);
                if (n == 0 && add == 0) continue;
                const int* sb = S.sbuf + k * A.spawn_cap;
                int* ls = S.lstk + k * kLocalCap;
                const unsigned lo = qget(P.ls_lo, k), hi = qget(P.ls_hi, k);
                const int size = (int)(hi - lo);
                // kLocalCap (128) >= 32 resumed parents: the overflow comes
                // from the stack and the children only
                const int over = size + n + add - kLocalCap;
                int from_sb = 0;
                if (over > 0) {
                    const int m1 = min(over, size);
                    if (m1 > 0) publish_stage(A, S, P, k, ls, lo, kLocalCap - 1, m1);
                    from_sb = min(over - m1, n);
                    if (from_sb > 0) publish_stage(A, S, P, k, sb, 0, 0xFFFFFFFFu, from_sb);
                    qset(P.ls_lo, k, lo + (unsigned)m1);
                }
                for (int e = from_sb + (int)lane; e < n; e += 32)
                    ls[(hi + (unsigned)(e - from_sb)) & (kLocalCap - 1)] = sb[e] & kIdMask;
                const unsigned h2 = hi + (unsigned)(n - from_sb);
                if ((mk >> lane) & 1u) ls[(h2 + (unsigned)__popc(mk & ((1u << lane) - 1u))) & (kLocalCap - 1)] = resumed;
                qset(P.ls_hi, k, h2 + (unsigned)add);
            }
            __syncwarp();   // local-stack entries written above are read below by other lanes
            if (kn < 0) {
                for (int kk = 0; kk < Q; ++kk) {
                    const int k = (P.cur_q + kk) % Q;
                    if (qget(P.ls_hi, k) != qget(P.ls_lo, k)) {
                        kn = k;
                        break;
                    }
                }
            }
            nb_next = 0;
            if (kn >= 0) {
                int* ls = S.lstk + kn * kLocalCap;
                const unsigned lo = qget(P.ls_lo, kn), hi = qget(P.ls_hi, kn);
                const int size = (int)(hi - lo);
                const int take = min(32, size);
                nb_next = take;
                if ((int)lane < take) {
                    next_tid = ls[(hi - (unsigned)take + lane) & (kLocalCap - 1)];
#ifdef GTAP_DEBUG_IDS
                    if (ld_cg(&A.dbg_live[next_tid]) != 1) GTAP_ERROR(A, ERR_POOL_SLOT_BUSY, next_tid, kn, 15, take);
#endif
                }
                qset(P.ls_hi, kn, hi - (unsigned)take);
                P.cur_q = kn;
            }
            __syncwarp();   // batch entries were read from the local stacks before they are published
            if (hungry > 0) {
                // keep one more batch in reserve so the next rounds stay full
                for (int k = 0; k < Q; ++k) {
                    const unsigned lo = qget(P.ls_lo, k), hi = qget(P.ls_hi, k);
                    const int size = (int)(hi - lo);
                    const int m = size - reserve;
                    if (m > 0) {
                        publish_stage(A, S, P, k, S.lstk + k * kLocalCap, lo, kLocalCap - 1, m);
                        qset(P.ls_lo, k, lo + (unsigned)m);
                    }
                }
            }
        }
        // the next batch's records (children this warp wrote, parents this
        // warp resumed) start on their way to the record stage: the copies
        // overlap the rest of the round end.  No other warp can take these
        // tasks any more, and this warp wrote or acquired their records: the
        // warp barrier orders every lane's stores before the copies, as it
        // orders them before the loads of a round that starts unstaged.
        staged = false;
        if (nb_next > 0 && S.rstage != nullptr) {
            __syncwarp();
            if ((int)lane < nb_next && (unsigned)next_tid < (unsigned)A.total_ids) {
                const char* rec = A.records + (size_t)next_tid * A.rec_stride;
                int4* st4 = S.rstage + lane * 3;
                cp_async16_cg(st4, rec);
                if (Prog::kFrameWords) {
                    cp_async16_cg(st4 + 1, rec + 16);
                    if (A.rec_stride >= 48) cp_async16_cg(st4 + 2, rec + 32);
                }
            }
            staged = true;
        }
        // (5) publication of the deque entries staged above (its own fence:
        //     the slot stores, and the records when nothing joined)
        publish_commit(A, S, P, false);
        GTAP_PHASE_MARK(ph4);
        GTAP_PHASE_ADD(13, ph3b, ph4);
        // (6) per-root accounting of finishes and values (creations were
        //     charged in (0)), one leader per distinct root
        if (one_root) {
            // every task of the round belongs to one root: warp sums, lane 0 books them
            const unsigned value = active ? (unsigned)S.l_value[lane] : 0u;
            const int w_sum = (Prog::kJoinSum && A.join_walk > 0) ? (int)__reduce_add_sync(0xffffffffu, (unsigned)walked) : 0;
            const int f_sum = __popc(fin) + w_sum;
            const int v_sum = (int)__reduce_add_sync(0xffffffffu, value);
            if (lane == 0) {
                if (v_sum) atomicAdd(reinterpret_cast<unsigned long long*>(&A.results[r0].value),
                                     (unsigned long long)(long long)v_sum);
                account_root(A, S, r0, 0, f_sum);
                if (S.nbal > 1) age_bal(A, S);
                else S.bal[0].touched = 0;
            }
            __syncwarp();
        } else {
            const int value = active ? S.l_value[lane] : 0;
            int f_sum = 0, v_sum = 0;
            if (active) {
                f_sum = __popc(fin & grp);
                if (Prog::kJoinSum && A.join_walk > 0) f_sum += (int)__reduce_add_sync(grp, (unsigned)walked);
                v_sum = (int)__reduce_add_sync(grp, (unsigned)value);
            }
            const bool leader = active && ((unsigned)__ffs(grp) - 1u == lane);
            unsigned leaders = __ballot_sync(0xffffffffu, leader);
            __syncwarp();
            while (leaders) {
                const unsigned l = (unsigned)__ffs(leaders) - 1u;
                if (lane == l) {
                    if (v_sum) atomicAdd(reinterpret_cast<unsigned long long*>(&A.results[my_root].value),
                                         (unsigned long long)(long long)v_sum);
                    account_root(A, S, my_root, 0, f_sum);
                }
                __syncwarp();
                leaders &= leaders - 1u;
            }
            if (lane == 0) age_bal(A, S);
            __syncwarp();
        }
        __syncwarp();
        if (lane == 0) {
            for (int k = 0; k < queue_count<QM>(A); ++k) S.cnt[k] = 0;
            S.st[GTAP_STAT_EXECUTIONS] += (unsigned long long)nb;
            S.st[GTAP_STAT_ROUNDS] += 1;
        }
        const unsigned created_all = __reduce_add_sync(0xffffffffu, (unsigned)(active ? S.l_created[lane] : 0));
        if (lane == 0) S.st[GTAP_STAT_TASKS] += created_all;
#ifndef GTAP_PHASE_TIMERS
        if (Prog::kJoinSum && A.join_walk > 0) {
            const unsigned walked_all = __reduce_add_sync(0xffffffffu, (unsigned)walked);
            if (lane == 0) S.st[GTAP_STAT_JOIN_FINISHES] += walked_all;
        }
#endif
        GTAP_PHASE_MARK(ph5);
        GTAP_PHASE_ADD(14, ph4, ph5);
        // (6) id cache
        id_cache_maintain(A, S);
        GTAP_PHASE_MARK(ph6);
        GTAP_PHASE_ADD(15, ph5, ph6);
        nb = nb_next;
        my_tid = next_tid;
        next_tid = -1;
        src_kind = 0;
        // periodic abort / watchdog check while busy
        if ((++round & 63) == 0) {
            int stop = 0;
            if (lane == 0) {
                if (aborted(A)) stop = 1;
                else if (watchdog_expired()) {
                    GTAP_ERROR(A, ERR_TIMEOUT, -1, -1, 1, 0);
                    stop = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, stop, 0)) break;
        }
    }
    rec_stage_wait();   // no copy outlives the loop
    if (lane == 0) flush_all_bal(A, S);
}

// One worker (warp): set up its WarpShared record S (this warp's staging
// buffer sbuf and local stack lstk given by the caller), run the loop, write
// its statistics.  initial_tid >= 0 starts lane 0 on that task (a task
// created before the loop, e.g. by the drop-in __gtap_push_initial_task).
template <class Prog, int QM>
__device__ __forceinline__ void thread_worker_run(const Arena& A, WarpShared& S, int worker, int* sbuf, int* lstk,
                                                  int initial_tid, int* lbuf = nullptr, int4* rstage = nullptr) {
    const unsigned lane = lane_id();
    if (lane == 0) {
        S.worker = worker;
        S.sbuf = sbuf;
        S.lstk = lstk;
        S.lbuf = lbuf;
        S.rstage = rstage;
        for (int k = 0; k < kMaxQueues; ++k) S.cnt[k] = 0;
        S.alloc_last = 0;
        S.alloc_pos = 0;
        S.freed_n = 0;
        S.nbal = 0;
        S.prof_h = 0;
        S.prof_w = 0;
        for (int i = 0; i < GTAP_STAT_COUNT; ++i) S.st[i] = 0;
    }
    // first ids come from the private range
    const int first = min(64, A.ids_per_worker);
    const int range = A.id_base + worker * A.ids_per_worker;
    S.l_pend[lane] = -1;
    if ((int)lane < first) S.avail[lane] = range + (int)lane;
    if ((int)lane + 32 < first) S.avail[lane + 32] = range + (int)lane + 32;
    if (lane == 0) {
        S.avail_head = 0;
        S.avail_n = first;
        S.bump = first;
    }
    __syncwarp();
    worker_loop<Prog, QM>(A, S, initial_tid);
    __syncwarp();
    if ((int)lane < GTAP_STAT_COUNT) A.stats[(size_t)worker * GTAP_STAT_COUNT + lane] = S.st[lane];
}

// Kernel body: warps_per_block WarpShared records + staging buffers in dynamic
// smem, then (programs with warp leaves) A.leaf_buf + 1 leaf buffers per warp,
// or (A.rec_prefetch, programs without them) a record stage of
// kRecStageBytes + 16 per warp.  The leaf buffers (2 KB or more a warp) double
// as the record stage: the stage is filled at a round's end and read when the
// next round starts, the leaf buffers only in between.
template <class Prog, int QM>
__device__ __forceinline__ void thread_worker_body(const Arena& A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wib = threadIdx.x >> 5;
    WarpShared* ws = reinterpret_cast<WarpShared*>(smem_raw);
    int* sb_base = reinterpret_cast<int*>(smem_raw + sizeof(WarpShared) * A.warps_per_block);
    int* ls_base = sb_base + (size_t)A.warps_per_block * A.num_queues * A.spawn_cap;
    int* lb_base = ls_base + (size_t)A.warps_per_block * A.num_queues * kLocalCap;
    const bool leaves = Prog::kLeafKeys && A.leaf_buf;
    int* lbuf = leaves ? lb_base + (size_t)wib * (A.leaf_buf + 1) * Prog::kLeafKeys : nullptr;
    int4* rstage = nullptr;
    if (A.rec_prefetch) {
        char* st = leaves ? reinterpret_cast<char*>(lbuf)
                          : reinterpret_cast<char*>(lb_base) + (size_t)wib * (kRecStageBytes + 16);
        rstage = reinterpret_cast<int4*>((reinterpret_cast<uintptr_t>(st) + 15) & ~(uintptr_t)15);
    }
    thread_worker_run<Prog, QM>(A, ws[wib], blockIdx.x * A.warps_per_block + wib,
                            sb_base + (size_t)wib * A.num_queues * A.spawn_cap,
                            ls_base + (size_t)wib * A.num_queues * kLocalCap, -1, lbuf, rstage);
}


// The arena descriptor stays in the kernel's parameter (constant) space:
// __grid_constant__ lets the scheduler take its address without the compiler
// copying its 400-odd bytes into every thread's local memory, where each field
// read would be a local load that mostly misses L1.
// At most kFullKernelThreads threads per block and 72 registers a thread:
// with 128-thread blocks seven workers' blocks fit an SM by registers (88
// unbounded registers allowed five), which runs the mix's fib and n-queens
// tasks faster than the few spills cost the sort paths.
constexpr int kFullKernelThreads = 896;
template <class Prog, int QM>
__global__ void __launch_bounds__(kFullKernelThreads, 1) thread_worker_kernel(const __grid_constant__ Arena A) {
    thread_worker_body<Prog, QM>(A);
}

// At most 64 registers per thread: any block size up to 1024 fits, and the
// light program reaches 32 resident warps per SM.
template <class Prog, int QM>
__global__ void __launch_bounds__(1024, 1) thread_worker_kernel_lb(const __grid_constant__ Arena A) {
    thread_worker_body<Prog, QM>(A);
}

}  // namespace gtap
