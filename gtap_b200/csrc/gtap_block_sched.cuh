// gtap_block_sched.cuh -- block-cooperative mode: one task = one CUDA block.
//
// Reference (paths relative to the reference project root):
//   BlockTaskQueue {queue[], top, bottom}     runtime/detail/block/gtap_runtime_block.cuh:22-26
//   pop :327-361 / steal :363-393 / push :395-438  (Chase-Lev per block, one task per steal)
//   __gtap_set_state_for_join_block :458-479, notify_parent :501-513, __gtap_finish_task :516-540
//   __gtap_spawn_task :542-575 (any thread of the block may spawn)
//   __gtap_execute_task_loop_device_impl :605-768 (continuation first: the resumed
//     parent, else the newest child, runs next on the same block)
//   block id pool                              runtime/detail/block/gtap_block_core.cuh:100-136
//
// The same arena as thread mode (task records, per-worker deques with the
// packed (tag | bottom | top) control word, the overflow and recycled-id
// rings, per-root outstanding counters), with one worker per block:
//   * warp 0 schedules: it acquires the next task (continuation, own deque
//     LIFO, one steal from the fullest of probe_width random victims, overflow
//     queue, a new root), and after the body it charges the children to their
//     root, publishes them and books the finish;
//   * all threads run the body; any thread may spawn: children are staged in
//     shared memory and published after the body (one fence, one add);
//   * the children a task creates are charged to its root before any of them
//     is published, the finish after the joins: a root completes exactly when
//     its counter returns to zero;
//   * the id cache is a shared-memory stack refilled between tasks from the
//     block's private range, the recycled-id ring and the never-used ids.
#pragma once
#include "gtap_programs.cuh"

namespace gtap {

constexpr int kBStage = 512;         // children staged per execution in shared memory
constexpr int kBAvail = 256;         // free ids cached per block
constexpr int kBAvailLow = 96;       // refill below this many
constexpr int kBMaxThreads = 512;    // threads per block in block mode (a leaf task's width)
constexpr int kBBal = 4;             // roots with a pre-charged balance per block
constexpr int kBRel = 64;            // ids released by task code in one execution, returned at round end
constexpr int kBChunk = 256;         // credit taken from a root's counter at a time

struct BlockShared {
    // the task this execution runs (written by warp 0 before the body)
    int task, kind, state, flags, parent, root;
    int4 w0, w1;                     // the frame's first 32 bytes
    unsigned long long fn;           // task function (programs with a function table)
    // spawn bookkeeping of this execution
    int nstaged;                     // children staged (beyond kBStage: waited per thread)
    int spawned;                     // children that join this task, since its last taskwait
    int suspended;                   // the body stopped at a taskwait with children outstanding
    int finished;
    long long value;                 // contributions to the root's value
    int next;                        // task to run next (continuation first), -1 none
    unsigned long long dq_word;      // this block's deque control word as last seen: tag and bottom exact
                                     // (only the owner moves them), top possibly behind (thieves move it)
    int pre_task;                    // the task whose record round end already loaded into the fields above
    int stop;
    int worker;
    int prof_h, prof_w;              // samples written to this block's profile timelines
    int having;                      // profile: the block holds a task (since its last idle poll)
    // id cache
    int avail_n;
    int bump;                        // next id of the private range
    int bump_end;
    int avail[kBAvail];
    int staged[kBStage];
    int pend[kBMaxThreads];          // per thread: a detached child past kBStage whose frame is being written
    int nrel;                        // ids task code released this execution (bt_release_deferred)
    int rel[kBRel];
    unsigned long long st[GTAP_STAT_COUNT];
    // pre-charged balances: the block holds credit[i] units of root bal_root[i]'s
    // outstanding count; finishes add to it, creations draw on it
    int nbal;
    int bal_root[kBBal];
    int bal_touched[kBBal];
    long long bal_credit[kBBal];
};

// ---------------------------------------------------------------------------
// single-thread pop from the recycled-id pool (the warp version needs all
// 32 lanes); -1 when the pool is empty
// ---------------------------------------------------------------------------
static __device__ int pool_pop_one(const Arena& A, const Ring& r) {
    const unsigned cap = 1u << r.cap_log2;
    for (int attempt = 0; attempt < 64; ++attempt) {
        unsigned h = 0;
        if (pool_claim(r, 1u, h) == 1u) {
            for (int spins = 0; spins <= (1 << 20); ++spins) {
                const unsigned long long w = ld_acquire(&r.slots[h & (cap - 1)]);
                if (ring_word_ready(w, h, r.cap_log2)) return ring_word_value(w);
                __nanosleep(64);
            }
            GTAP_ERROR(A, ERR_TIMEOUT, -1, -1, (int)h, 0);
            return -1;
        }
        const unsigned t = ld_relaxed(r.tail), hh = ld_relaxed(r.head);
        if (t == hh || t - hh > cap) return -1;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// task ABI of block mode (called by the task bodies)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int bt_state(const BlockShared& S) { return S.state; }
__device__ __forceinline__ const gtap_root& bt_root(const Arena& A, const BlockShared& S) { return A.roots[S.root]; }

// Any thread.  The shared cache first; when it runs dry inside one execution,
// a recycled id, else a never-used one.
__device__ __forceinline__ int bt_alloc_id(const Arena& A, BlockShared& S) {
    const int k = atomicSub(&S.avail_n, 1) - 1;
    if (k >= 0) return S.avail[k];
    const int v = pool_pop_one(A, A.idpool);
    if (v >= 0) return v;
    const unsigned f = atomicAdd(A.fresh_next, 1u);
    if (f < (unsigned)A.total_ids) return (int)f;
    GTAP_ERROR(A, ERR_POOL_EXHAUSTED, S.task, -1, (int)f, A.total_ids);
    return A.total_ids;
}

// A detached child past the staging list, once its frame is written (by the
// thread that spawned it): fence, then the overflow queue.
__device__ __forceinline__ void bt_push_pending(const Arena& A, BlockShared& S, int id) {
    fence_acq_rel();
    ring_push_one(A.overflow, id);
    atomicAdd(&S.st[GTAP_STAT_OVERFLOW_PUSHES], 1ull);
}

// Any thread.  The caller writes the child's frame after this returns; the
// child is published after the body (reference contract of __gtap_spawn_task).
__device__ __forceinline__ void* bt_spawn(const Arena& A, BlockShared& S, int kind, int* child_count, int* out_tid,
                                          bool retain, bool detached) {
    const int id = bt_alloc_id(A, S);
    if (out_tid) *out_tid = id;
    if (id >= A.total_ids) return frame_of(A, A.total_ids);   // allocation failed; error recorded
    int4 hw;
    hw.x = (int)((unsigned)kind << 16 | (unsigned)(retain ? kFlagRetain : 0) << 24);
    hw.y = detached ? -1 : S.task;
    hw.z = 0;
    hw.w = S.root;
    *reinterpret_cast<int4*>(hdr_of(A, id)) = hw;
    const int k = atomicAdd(&S.nstaged, 1);
    if (k < kBStage) {
        S.staged[k] = id;
    } else if (detached) {
        // charged to the root now; pushed at this thread's next spawn or when
        // the body returns, once its frame is written
        red_add_relaxed(&A.outstanding[S.root], 1ll);
        red_add_relaxed(reinterpret_cast<long long*>(&A.results[S.root].tasks), 1ll);
        atomicAdd(&S.st[GTAP_STAT_TASKS], 1ull);
        const int prev = S.pend[threadIdx.x];
        S.pend[threadIdx.x] = id;
        if (prev >= 0) bt_push_pending(A, S, prev);
    } else {
        GTAP_ERROR(A, ERR_SPAWN_BUFFER_OVERFLOW, S.task, -1, k, kBStage);
    }
    if (!detached) atomicAdd(&S.spawned, 1);
    if (child_count) ++*child_count;
    return frame_of(A, id);
}

// All threads (block-uniform).  taskwait: the children spawned since the last
// one become this task's join count; true if the task must suspend.  The
// header is written before any of the children is published.  then_finish:
// the task's code after this taskwait only finishes, so the block that
// completes the join books the finish instead of running the task again.
__device__ __forceinline__ bool bt_join(const Arena& A, BlockShared& S, int next_state, bool then_finish = false) {
    __syncthreads();
    const int n = S.spawned;
    __syncthreads();
    if (threadIdx.x == 0) {
        S.state = next_state;
        S.spawned = 0;
        if (n > 0) {
            TaskHeader* h = hdr_of(A, S.task);
            h->state = (uint16_t)next_state;
            if (then_finish) h->flags = (uint8_t)(S.flags | kFlagJoinFinish);
            h->join = n & kJoinCountMask;
            S.suspended = 1;
        }
    }
    __syncthreads();
    return n > 0;
}

// All threads (block-uniform): the task is done.
__device__ __forceinline__ void bt_finish(BlockShared& S) {
    if (threadIdx.x == 0) S.finished = 1;
}

// One thread: the task's result, into its parent's frame at byte offset
// `slot`, or into the root result for a root task.
__device__ __forceinline__ void bt_return_i64(const Arena& A, const BlockShared& S, int slot, long long v) {
    if (S.parent >= 0) *reinterpret_cast<long long*>(reinterpret_cast<char*>(frame_of(A, S.parent)) + slot) = v;
    else A.results[S.root].value = v;
}
__device__ __forceinline__ void bt_return_i32(const Arena& A, const BlockShared& S, int slot, int v) {
    if (S.parent >= 0) *reinterpret_cast<int*>(reinterpret_cast<char*>(frame_of(A, S.parent)) + slot) = v;
    else A.results[S.root].value = v;
}
// Any thread: add to the root's value (n-queens counts).
__device__ __forceinline__ void bt_add_value(BlockShared& S, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&S.value), (unsigned long long)v);
}

// Any thread: a retained child's id, once its frame has been read.  It goes
// back at round end, after the barrier that ends the body, so no thread of
// the block can still be reading the frame; past kBRel per execution it goes
// to the recycled-id ring at once (the caller has finished reading it).
__device__ __forceinline__ void bt_release_deferred(const Arena& A, BlockShared& S, int id) {
    if ((unsigned)id >= (unsigned)A.total_ids) return;
    const int k = atomicAdd(&S.nrel, 1);
    if (k < kBRel) {
        S.rel[k] = id;
    } else {
        fence_acq_rel();
        ring_push_one(A.idpool, id);
    }
}

// ---------------------------------------------------------------------------
// per-root balances (lane 0 of warp 0).  A root's counter = its live tasks +
// the credit blocks hold for it, so it reaches zero exactly when the last task
// has finished and every block has returned its credit; the global counter is
// touched once per kBChunk creations and once per flush instead of per task.
// ---------------------------------------------------------------------------
static __device__ void bt_bal_flush(const Arena& A, BlockShared& S, int i) {
    const long long c = S.bal_credit[i];
    const int r = S.bal_root[i];
    --S.nbal;
    S.bal_root[i] = S.bal_root[S.nbal];
    S.bal_credit[i] = S.bal_credit[S.nbal];
    S.bal_touched[i] = S.bal_touched[S.nbal];
    if (c != 0) outstanding_add(A, r, -c);
}
static __device__ int bt_bal_slot(const Arena& A, BlockShared& S, int r) {
    for (int i = 0; i < S.nbal; ++i)
        if (S.bal_root[i] == r) return i;
    if (S.nbal == kBBal) bt_bal_flush(A, S, 0);
    const int i = S.nbal++;
    S.bal_root[i] = r;
    S.bal_credit[i] = 0;
    S.bal_touched[i] = 0;
    return i;
}
// n creations for root r, before any of them is published
static __device__ void bt_charge(const Arena& A, BlockShared& S, int r, int n) {
    const int i = bt_bal_slot(A, S, r);
    S.bal_touched[i] = 1;
    long long c = S.bal_credit[i] - n;
    if (c < 0) {
        red_add_relaxed(&A.outstanding[r], (long long)kBChunk - c);
        c = kBChunk;
    }
    S.bal_credit[i] = c;
}
// one finish of root r
static __device__ void bt_credit(const Arena& A, BlockShared& S, int r) {
    const int i = bt_bal_slot(A, S, r);
    S.bal_touched[i] = 1;
    S.bal_credit[i] += 1;
}
// after a task: balances of roots this task did not touch go back, so that
// completions are not held up by blocks busy elsewhere
static __device__ void bt_bal_age(const Arena& A, BlockShared& S) {
    for (int i = S.nbal - 1; i >= 0; --i) {
        if (S.bal_touched[i]) S.bal_touched[i] = 0;
        else bt_bal_flush(A, S, i);
    }
}
static __device__ void bt_bal_flush_all(const Arena& A, BlockShared& S) {
    while (S.nbal > 0) bt_bal_flush(A, S, S.nbal - 1);
}

// ---------------------------------------------------------------------------
// profile timelines (reference runtime/detail/block/gtap_profile_block.cuh):
// one row per block; "having task" spans open when the block finds work after
// an idle poll and close at the next idle poll, "working" spans cover each
// task execution (thread 0 writes both)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bt_prof_having(const Arena& A, BlockShared& S) {
    if (A.prof_cap > 0 && S.prof_h < A.prof_cap) {
        A.prof_having[(size_t)S.worker * A.prof_cap + S.prof_h] = (long long)global_ns();
        S.prof_h++;
    }
}
__device__ __forceinline__ void bt_prof_working(const Arena& A, BlockShared& S) {
    if (A.prof_cap > 0 && S.prof_w < A.prof_cap) {
        const size_t i = (size_t)S.worker * A.prof_cap + S.prof_w;
        A.prof_working[i] = (long long)global_ns();
        A.prof_tasks[i] = 1;
        S.prof_w++;
    }
}

// ---------------------------------------------------------------------------
// scheduling (warp 0; lane 0 unless noted)
// ---------------------------------------------------------------------------
// Owner pop, newest first (reference pop :327-361, as one CAS on the control
// word).  The CAS starts from the cached word: its size can only overstate the
// deque's (thieves only advance top), so an empty cache means an empty deque,
// and a stale top fails the CAS, which returns the current word.  The slot
// load goes out with the CAS: this block wrote that slot, and the value is
// used only if the CAS claims it.  One round trip when no thief interferes.
static __device__ int bt_pop_own(const Arena& A, BlockShared& S) {
    unsigned long long* c = dq_ctl_ptr(A, 0, S.worker);
    unsigned long long wv = S.dq_word;
    for (int i = 0; i < 16; ++i) {
        if (dq_size(wv) == 0) break;
        const int id = ld_relaxed(dq_slot_ptr(A, 0, S.worker, dq_bottom(wv) - 1u));
        const unsigned long long nw = dq_owner_pop(wv, 1);
        const unsigned long long old = atom_cas_acquire(c, wv, nw);
        if (old == wv) {
            S.dq_word = nw;
            S.st[GTAP_STAT_POPS] += 1;
            return id;
        }
        wv = old;
    }
    S.dq_word = wv;
    return -1;
}

// One task from the top of the fullest of probe_width random victims (all
// lanes of warp 0; reference steal :363-393 probes one victim).
static __device__ int bt_steal(const Arena& A, BlockShared& S, unsigned& rng) {
    const unsigned lane = lane_id();
    const int W = A.num_workers;
    if (W < 2) return -1;
    int victim = -1;
    unsigned long long wv = 0;
    unsigned sz = 0;
    if ((int)lane < A.probe_width) {
        int v = (int)(xorshift32(rng) % (unsigned)(W - 1));
        if (v >= S.worker) ++v;
        victim = v;
        wv = ld_acquire(dq_ctl_ptr(A, 0, v));
        sz = dq_size(wv);
    }
    unsigned key = (sz << 5) | (31u - lane);
    if (sz > (1u << 21)) key = 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if (lane == 0) S.st[GTAP_STAT_STEAL_ATTEMPTS] += 1;
    if ((key >> 5) == 0) return -1;
    const int src = 31 - (int)(key & 31u);
    victim = __shfl_sync(0xffffffffu, victim, src);
    wv = __shfl_sync(0xffffffffu, wv, src);
    int got = -1;
    if (lane == 0) {
        unsigned long long* c = dq_ctl_ptr(A, 0, victim);
        for (int attempt = 0; attempt < 3; ++attempt) {
            const unsigned size = dq_size(wv);
            if (size == 0 || size > (1u << 20)) break;
            const unsigned t = dq_top(wv);
            // acquire: the slot is read before the CAS that claims it lands
            const int id = ld_acquire(dq_slot_ptr(A, 0, victim, t));
            const unsigned long long old = atom_cas_acquire(c, wv, dq_with_top(wv, t + 1u));
            if (old == wv) {
                S.st[GTAP_STAT_STEAL_SUCCESSES] += 1;
                S.st[GTAP_STAT_STOLEN_TASKS] += 1;
                got = id;
                break;
            }
            wv = old;
        }
    }
    return __shfl_sync(0xffffffffu, got, 0);
}

// A new root, claimed from the table (batch) or the published ring (serve);
// its task is created here and runs on this block at once.
template <class Prog>
static __device__ int bt_admit(const Arena& A, BlockShared& S) {
    unsigned limit = (A.mode == 2) ? ld_acquire(A.published) : (unsigned)A.n_roots;
    const unsigned fresh = ld_relaxed(A.fresh_next);
    const unsigned pool = ld_relaxed(A.idpool.tail) - ld_relaxed(A.idpool.head);
    const long long free_ids = (long long)A.total_ids - (long long)fresh + (long long)pool;
    if (free_ids < (long long)A.admit_watermark) limit = 0;
    if (A.max_inflight > 0) {
        const unsigned cap = ld_relaxed(A.completed) + (unsigned)A.max_inflight;
        if (cap < limit) limit = cap;
    }
    int idx = -1;
    for (int attempt = 0; attempt < 8; ++attempt) {
        const unsigned c = ld_relaxed(A.next_root);
        if (c >= limit) break;
        if (atom_cas_relaxed(A.next_root, c, c + 1u) == c) {
            idx = (int)c;
            break;
        }
    }
    if (idx < 0) return -1;
    const int slot = (A.mode == 2) ? (int)((unsigned)idx % (unsigned)A.n_roots) : idx;
    const gtap_root& rd = A.roots[slot];
    int id = bt_alloc_id(A, S);
    if (id >= A.total_ids) id = A.total_ids;   // error recorded; the launch aborts
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
    int4 hw;
    hw.x = (int)((unsigned)kind << 16);
    hw.y = -1;
    hw.z = 0;
    hw.w = slot;
    *reinterpret_cast<int4*>(hdr_of(A, id)) = hw;
    if (valid) Prog::init_root(A, rd, frame_of(A, id));
    gtap_root_result* res = &A.results[slot];
    res->value = 0;
    res->tasks = 1;
    res->t_done_ns = 0;
    res->t_admit_ns = global_ns();
    res->index = idx;
    res->status = GTAP_ROOT_RUNNING;
    atom_add_acq_rel(&A.outstanding[slot], 1ll);
    S.st[GTAP_STAT_TASKS] += 1;
    return id;
}

// Warp 0: top the id cache up between tasks -- private range first, then
// recycled ids, then never-used ones in batches of 32.
static __device__ void bt_refill_ids(const Arena& A, BlockShared& S) {
    const unsigned lane = lane_id();
    int n = S.avail_n;
    if (n < 0) n = 0;
    if (n >= kBAvailLow) {
        if (lane == 0) S.avail_n = n;
        __syncwarp();
        return;
    }
    for (int round = 0; round < 8 && n < kBAvail - 32; ++round) {
        int got = 0;
        const int priv = S.bump_end - S.bump;
        if (priv > 0) {
            got = min(32, priv);
            if ((int)lane < got) S.avail[n + lane] = S.bump + (int)lane;
            __syncwarp();
            if (lane == 0) S.bump += got;
        } else {
            int v = -1;
            got = ring_pop_warp(A, A.idpool, 32, &v, true);
            if ((int)lane < got) S.avail[n + lane] = v;
            if (got == 0) {
                unsigned f = 0;
                if (lane == 0) f = atomicAdd(A.fresh_next, 32u);
                f = __shfl_sync(0xffffffffu, f, 0);
                if (f >= (unsigned)A.total_ids) break;   // exhausted: spawns record the error
                got = (int)min(32u, (unsigned)A.total_ids - f);
                if ((int)lane < got) S.avail[n + lane] = (int)(f + lane);
            }
        }
        __syncwarp();
        n += got;
    }
    if (lane == 0) S.avail_n = n;
    __syncwarp();
}

// lane 0: a finished task's id goes back to the cache (or the recycled-id
// ring) unless its parent still reads the task's frame
static __device__ void bt_release_id(const Arena& A, BlockShared& S, int id, unsigned flags) {
    if (flags & kFlagRetain) return;
    if (S.avail_n < kBAvail && S.avail_n >= 0) S.avail[S.avail_n++] = id;
    else ring_push_one(A.idpool, id);
}

// Warp 0, after the body: charge, publish, join, finish, release.
template <class Prog>
static __device__ void bt_round_end(const Arena& A, BlockShared& S) {
    const unsigned lane = lane_id();
    const int t = S.task;
    const int root = S.root;
    const int n_st = min(S.nstaged, kBStage);
    const bool finished = S.finished != 0 || S.suspended == 0;
    // the newest child usually runs next on this block: lanes 1-3 load its
    // record now, overlapping the fence and the join below (this block wrote
    // it, before the barrier that precedes round end)
    const int kept = n_st > 0 ? S.staged[n_st - 1] : -1;
    int4 pre = make_int4(0, 0, 0, 0);
    unsigned long long pre_fn = 0;
    if (kept >= 0 && lane >= 1 && lane <= 3) pre = ld_data_v4(A.records + (size_t)kept * A.rec_stride + 16 * (lane - 1));
    if (Prog::kFuncTable && kept >= 0 && lane == 4) pre_fn = ld_data_u64(reinterpret_cast<const unsigned long long*>(A.funcs + kept));
    // (1) the round's value and its children count for the root before any
    //     child can be seen by another block
    if (lane == 0) {
        if (S.value) atomicAdd(reinterpret_cast<unsigned long long*>(&A.results[root].value),
                               (unsigned long long)S.value);
        if (n_st > 0) {
            bt_charge(A, S, root, n_st);
            red_add_relaxed(reinterpret_cast<long long*>(&A.results[root].tasks), (long long)n_st);
            S.st[GTAP_STAT_TASKS] += (unsigned long long)n_st;
        }
    }
    // (2) children of a task that returned without a taskwait are orphans
    if (finished && S.spawned > 0)
        for (int e = (int)lane; e < n_st; e += 32) hdr_of(A, S.staged[e])->parent = -1;
    // (3) the newest child runs next unless a parent resumes; the rest go to
    //     the deque (oldest at the top, where thieves take), or to the
    //     overflow queue when it is full
    int keep = (n_st > 0) ? 1 : 0;
    const int m = n_st - keep;   // a resumed parent may claim the kept child's place below
    unsigned b = 0;
    int direct = 0;
    unsigned long long* c = dq_ctl_ptr(A, 0, S.worker);
    if (m > 0) {
        // the cached control word: bottom exact, the size at most overstated
        // (a thief's steal may not be in it), so the room is never overstated
        const unsigned long long wv = S.dq_word;
        const unsigned cap = 1u << A.deque_cap_log2;
        const unsigned used = dq_size(wv);
        b = dq_bottom(wv);
        direct = (used + (unsigned)m > cap) ? (int)(cap - min(used, cap)) : m;
        for (int e = (int)lane; e < direct; e += 32) *dq_slot_ptr(A, 0, S.worker, b + (unsigned)e) = S.staged[e];
    }
    __syncwarp();
    // one fence orders the body's stores (the whole block's, through the
    // barrier before this), the records and the slots before what follows.
    // (For a finished task that publishes nothing, an acquire-release join
    // decrement in place of this fence and an acquire-only one measured
    // slower: 12.40 against 12.23 ms for 2^26 keys.)
    if (lane == 0) fence_acq_rel();
    __syncwarp();
    if (m > direct) {
        for (int base = direct; base < m; base += 32) {
            const int take = min(32, m - base);
            const int id = ((int)lane < take) ? S.staged[base + (int)lane] : 0;
            ring_push_warp(A, A.overflow, id, take);
        }
        if (lane == 0) S.st[GTAP_STAT_OVERFLOW_PUSHES] += (unsigned long long)(m - direct);
    }
    if (lane == 0) {
        if (direct > 0) {
            red_add_relaxed(c, (unsigned long long)direct << kPosBits);
            S.dq_word += (unsigned long long)direct << kPosBits;
            S.st[GTAP_STAT_PUBLISHED] += (unsigned long long)direct;
        }
        int next = kept;
        // ids the task code released (retained children it has read)
        for (int i = 0; i < min(S.nrel, kBRel); ++i) bt_release_id(A, S, S.rel[i], 0);
        if (finished) {
            // (4) the finish counts for the root; the id goes back unless the
            //     parent still reads this task's frame
            bt_release_id(A, S, t, S.flags);
            bt_credit(A, S, root);
            // (5) join: the last child resumes its parent on this block, or,
            //     when the parent's code after its taskwait only finishes,
            //     books that finish here and goes on to the grandparent
            int parent = S.parent;
            bool first = true;
            while (parent >= 0) {
                // The parent's flags, parent and root are final before any of
                // its children was published (bt_join writes the header
                // first), so the header load goes out together with the join
                // decrement: one round trip per level instead of two.
                const int4 ph = ld_cg_v4(hdr_of(A, parent));
                // past the first level this block publishes what it observed
                // through the previous join (the siblings' data) onwards
                const int old = first ? atom_add_acquire(&hdr_of(A, parent)->join, -1)
                                      : atom_add_acq_rel(&hdr_of(A, parent)->join, -1);
                first = false;
                if ((old & kJoinCountMask) != 1) break;
                const unsigned pflags = (unsigned)ph.x >> 24;
                if (!(pflags & kFlagJoinFinish)) {
                    if (next >= 0) {
                        // the kept child is published after all
                        ring_push_one(A.overflow, next);
                        S.st[GTAP_STAT_OVERFLOW_PUSHES] += 1;
                    }
                    next = parent;
                    break;
                }
                bt_release_id(A, S, parent, pflags);
                bt_credit(A, S, ph.w);
#ifndef GTAP_PHASE_TIMERS
                S.st[GTAP_STAT_JOIN_FINISHES] += 1;
#endif
                parent = ph.y;
            }
        }
        bt_bal_age(A, S);
        S.next = next;
        S.pre_task = (next >= 0 && next == kept) ? kept : -1;
        S.st[GTAP_STAT_EXECUTIONS] += 1;
        S.st[GTAP_STAT_ROUNDS] += 1;
    }
    __syncwarp();
    // the prefetched record becomes the next task's (orphan marking above
    // cleared its parent when this task returned without a taskwait)
    if (Prog::kFuncTable && kept >= 0 && S.pre_task == kept && lane == 4) S.fn = pre_fn;
    if (kept >= 0 && S.pre_task == kept && lane >= 1 && lane <= 3) {
        if (lane == 1) {
            const unsigned x = (unsigned)pre.x;
            S.state = (int)(x & 0xFFFFu);
            S.kind = (int)((x >> 16) & 0xFFu);
            S.flags = (int)(x >> 24);
            S.parent = (finished && S.spawned > 0) ? -1 : pre.y;
            S.root = pre.w;
        } else if (lane == 2) {
            S.w0 = pre;
        } else {
            S.w1 = pre;
        }
    }
    __syncwarp();
    bt_refill_ids(A, S);
}

// ---------------------------------------------------------------------------
// the persistent loop
// ---------------------------------------------------------------------------
// Profiling builds (-DGTAP_PHASE_TIMERS): thread 0 adds the clock64 cycles of
// each phase to statistics slots 10..15 (acquire, record load, body, pending
// children + barrier, round end, idle polls).
#ifdef GTAP_PHASE_TIMERS
#define GTAP_BPHASE(t) const long long t = clock64()
#define GTAP_BPHASE_ADD(slot, a, b) \
    do {                            \
        if (tid == 0) S.st[slot] += (unsigned long long)((b) - (a)); \
    } while (0)
#else
#define GTAP_BPHASE(t) \
    do {               \
    } while (0)
#define GTAP_BPHASE_ADD(slot, a, b) \
    do {                            \
    } while (0)
#endif

// initial_tid >= 0: this block starts with that task (one created before the
// loop, e.g. by the drop-in __gtap_push_initial_task).
template <class Prog>
__device__ void block_worker(const Arena& A, BlockShared& S, int* smem, int initial_tid = -1) {
    const int tid = threadIdx.x;
    const unsigned lane = lane_id();
    const bool w0 = tid < 32;
    if (tid == 0) {
        S.worker = blockIdx.x;
        S.next = initial_tid;
        S.dq_word = ld_relaxed(dq_ctl_ptr(A, 0, blockIdx.x));   // reset before the launch
        S.pre_task = -1;
        S.stop = 0;
        S.task = -1;
        S.bump = A.id_base + blockIdx.x * A.ids_per_worker;
        S.bump_end = S.bump + A.ids_per_worker;
        S.avail_n = 0;
        S.nbal = 0;
        S.prof_h = 0;
        S.prof_w = 0;
        S.having = 0;
        for (int i = 0; i < GTAP_STAT_COUNT; ++i) S.st[i] = 0;
    }
    for (int i = tid; i < kBMaxThreads; i += blockDim.x) S.pend[i] = -1;
    __syncthreads();
    if (w0) bt_refill_ids(A, S);
    unsigned rng = 0x9E3779B9u ^ (unsigned)(blockIdx.x * 2654435761u) ^ (lane * 0x85EBCA6Bu) ^ (unsigned)clock64();
    if (rng == 0) rng = 1;
    int backoff = 0;
    // watchdog (lane 0 of warp 0): a batch launch is bounded as a whole; a
    // serve session only while roots are outstanding and none completes
    unsigned long long t_watch = global_ns();
    unsigned seen_done = 0;
    int round = 0;
    bool idle = false;                       // thread 0: in an idle stretch
    unsigned long long idle_since = 0;       // thread 0: since when
    __syncthreads();
    for (;;) {
        GTAP_BPHASE(ph0);
        // ---- acquire (warp 0) ----
        if (w0) {
            int t = -1;
            if (lane == 0) {
                t = S.next;
                S.next = -1;
                if (t < 0) t = bt_pop_own(A, S);
            }
            t = __shfl_sync(0xffffffffu, t, 0);
            if (t < 0) t = bt_steal(A, S, rng);
            if (t < 0) {
                int v = -1;
                const int got = ring_pop_warp(A, A.overflow, 1, &v);
                v = __shfl_sync(0xffffffffu, v, 0);
                if (got) t = v;
            }
            if (lane == 0) {
                if (t < 0) t = bt_admit<Prog>(A, S);
                int stop = 0;
                if (t < 0) {
                    S.st[GTAP_STAT_IDLE_POLLS] += 1;
                    if (!idle) idle_since = global_ns();
                    idle = true;
                    bt_bal_flush_all(A, S);
                    if (S.having) {
                        bt_prof_having(A, S);
                        S.having = 0;
                    }
                    if (ld_acquire(A.done_flag) != 0 || aborted(A)) stop = 1;
                    if (A.mode == 2 && ld_relaxed(A.shutdown) != 0) {
                        const unsigned pub = ld_acquire(A.published);
                        if (ld_acquire(A.completed) >= pub && ld_relaxed(A.next_root) >= pub) stop = 1;
                    }
                    if (!stop) {
                        const unsigned long long now = global_ns();
                        if (A.mode == 2) {
                            const unsigned cdone = ld_relaxed(A.completed);
                            if (cdone != seen_done || cdone >= ld_relaxed(A.published)) {
                                seen_done = cdone;
                                t_watch = now;
                            }
                        }
                        if (now - t_watch > A.watchdog_ns) {
                            GTAP_ERROR(A, ERR_TIMEOUT, -1, -1, 2, 0);
                            stop = 1;
                        }
                    }
                    if (backoff < 6) ++backoff;
                    __nanosleep(32u << backoff);
                } else {
                    backoff = 0;
#ifndef GTAP_PHASE_TIMERS
                    if (idle) S.st[GTAP_STAT_IDLE_NS] += global_ns() - idle_since;
#endif
                    idle = false;
                    if (!S.having) {
                        bt_prof_having(A, S);
                        S.having = 1;
                    }
                    if ((++round & 63) == 0) {
                        if (aborted(A)) stop = 1;
                        else if (A.mode != 2 && global_ns() - t_watch > A.watchdog_ns) {
                            GTAP_ERROR(A, ERR_TIMEOUT, -1, -1, 3, 0);
                            stop = 1;
                        }
                    }
                }
#ifndef GTAP_PHASE_TIMERS
                if (stop && idle) S.st[GTAP_STAT_IDLE_NS] += global_ns() - idle_since;
#endif
                S.stop = stop;
                S.task = t;
                S.nrel = 0;
                S.nstaged = 0;
                S.spawned = 0;
                S.suspended = 0;
                S.finished = 0;
                S.value = 0;
            }
        }
        __syncthreads();
        GTAP_BPHASE(ph1);
        if (S.stop) break;
        const int t = S.task;
        if (t < 0) {
            GTAP_BPHASE_ADD(15, ph0, ph1);
            continue;
        }
        GTAP_BPHASE_ADD(10, ph0, ph1);
        // ---- record: header + first 32 frame bytes (already loaded by the
        //      last round end when this is the child it kept: every round end
        //      sets pre_task, and that child is the next task acquired) ----
        const bool preloaded = S.pre_task == t;
        if (Prog::kFuncTable && !preloaded && tid == 3) S.fn = ld_data_u64(reinterpret_cast<const unsigned long long*>(A.funcs + t));
        if (!preloaded && tid < 3) {
            const int4 v = ld_data_v4(A.records + (size_t)t * A.rec_stride + 16 * tid);
            if (tid == 0) {
                const unsigned x = (unsigned)v.x;
                S.state = (int)(x & 0xFFFFu);
                S.kind = (int)((x >> 16) & 0xFFu);
                S.flags = (int)(x >> 24);
                S.parent = v.y;
                S.root = v.w;
            } else if (tid == 1) {
                S.w0 = v;
            } else {
                S.w1 = v;
            }
        }
        __syncthreads();
        GTAP_BPHASE(ph2);
        GTAP_BPHASE_ADD(11, ph1, ph2);
        // ---- body (all threads) ----
        if (tid == 0) bt_prof_working(A, S);
        Prog::exec(A, S, t, smem);
        GTAP_BPHASE(ph3);
        GTAP_BPHASE_ADD(12, ph2, ph3);
        // detached children past the staging list: their frames are written
        // by the threads that spawned them, which publish them
        {
            const int pend = S.pend[tid];
            if (pend >= 0) {
                S.pend[tid] = -1;
                bt_push_pending(A, S, pend);
            }
        }
        __syncthreads();
        GTAP_BPHASE(ph4);
        GTAP_BPHASE_ADD(13, ph3, ph4);
        if (w0) bt_round_end<Prog>(A, S);
        if (tid == 0) bt_prof_working(A, S);
        __syncthreads();
        GTAP_BPHASE(ph5);
        GTAP_BPHASE_ADD(14, ph4, ph5);
    }
    __syncthreads();
    if (tid == 0) bt_bal_flush_all(A, S);
    if (w0 && (int)lane < GTAP_STAT_COUNT) A.stats[(size_t)S.worker * GTAP_STAT_COUNT + lane] = S.st[lane];
}

}  // namespace gtap
