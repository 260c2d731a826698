/*
 * gtap_types.h -- plain C types and constants of the B200 GTaP runtime, shared
 * by the C ABI (gtap.h), the device code and the drop-in task-ABI header
 * (gtap_thread.cuh).  No function declarations: gtap_thread.cuh defines the
 * reference's host functions (gtap_initialize() and friends, returning
 * cudaError_t), whose names the C ABI in gtap.h also uses with other types.
 */
#ifndef GTAP_B200_TYPES_H
#define GTAP_B200_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* error codes: 0..8 keep runtime/detail/common/gtap_runtime_error.cuh:7-18 */
/* ------------------------------------------------------------------------ */
enum {
    GTAP_ERROR_NONE = 0,
    GTAP_ERROR_INVALID_QUEUE_IDX = 1,
    GTAP_ERROR_INVALID_QUEUE_IDX_AFTER_JOIN = 2,
    GTAP_ERROR_QUEUE_OVERFLOW = 3,
    GTAP_ERROR_RESULT_HANDLE_OVERFLOW = 4,
    GTAP_ERROR_TASK_ID_POOL_SLOT_BUSY = 5,
    GTAP_ERROR_TASK_ID_POOL_LOW_HEADROOM = 6,
    GTAP_ERROR_GENERATED_TASK_ID_BUFFER_OVERFLOW = 7,
    GTAP_ERROR_INVALID_TASKWAIT = 8,
    GTAP_ERROR_TIMEOUT = 9,           /* NEW: a bounded wait or the launch watchdog ran out */
    GTAP_ERROR_INVALID_KIND = 10,     /* NEW: unknown task kind in a root descriptor */
    GTAP_ERROR_INVALID_ARGUMENT = 11, /* NEW: host-side argument check */
    GTAP_ERROR_NOT_INITIALIZED = 12,  /* NEW */
    GTAP_ERROR_BUSY = 13,             /* NEW: a serve session is running */
    GTAP_ERROR_COUNT
};

/* Device-written error report (first error wins); layout of the reference's
 * GTapRuntimeErrorReport, runtime/detail/common/gtap_runtime_error.cuh:20-30. */
typedef struct GtapErrorReport {
    int valid;
    int code;
    int src_line;
    int block_idx;
    int thread_idx;
    int tid;
    int queue_idx;
    int value;
    int limit;
} GtapErrorReport;

/* Legacy result handle, runtime/detail/thread/gtap_thread_core.cuh:62-67. */
typedef struct gtap_result_handle {
    int child_tid;
    int kind;
    int next;
    int pad;
    void* lhs_addr;
} gtap_result_handle;

/* ------------------------------------------------------------------------ */
/* launch configuration (NEW: the reference fixes these with -D macros,     */
/* runtime/detail/common/gtap_config.cuh:6-28, gtap_runtime_thread.cuh:10-24)*/
/* ------------------------------------------------------------------------ */
enum { GTAP_MODE_THREAD = 0, GTAP_MODE_BLOCK = 1 };
enum { GTAP_VICTIM_RANDOM = 0, GTAP_VICTIM_LAST_SUCCESS = 1, GTAP_VICTIM_PROBE_MAX = 2 };

typedef struct gtap_config {
    int32_t mode;            /* GTAP_MODE_THREAD (1 task = 1 thread) or GTAP_MODE_BLOCK (1 task = 1 block) */
    int32_t grid;            /* blocks; 0 = one persistent wave sized from the SM count */
    int32_t block;           /* threads per block, multiple of 32 (GTAP_BLOCK_SIZE) */
    int32_t num_queues;      /* EPAQ queues 1..4 (GTAP_NUM_QUEUES) */
    int32_t deque_capacity;  /* per worker per queue, power of two (GTAP_MAX_TASKS_PER_WARP / Q) */
    int32_t steal_batch;     /* tasks moved by one steal, 1..32 (reference: up to 32) */
    int32_t victim_policy;   /* GTAP_VICTIM_* (reference: uniform random) */
    int32_t probe_width;     /* victims probed in parallel per steal attempt, 1..32 */
    int32_t spawn_capacity;  /* children staged per queue per worker and round (GTAP_MAX_CHILD_TASKS x 32) */
    int32_t ids_per_worker;  /* private id range per worker */
    int64_t total_ids;       /* task records in the arena (<= 2^27) */
    int32_t frame_bytes;     /* largest task frame in bytes (__gtap_auto_task_data_size) */
    int32_t admit_batch;     /* roots an idle worker claims at once */
    int64_t watchdog_ms;     /* hard wall-clock limit per launch (serve mode: per stretch with roots
                                outstanding and none completing); the kernel returns GTAP_ERROR_TIMEOUT */
    int32_t profile_samples; /* per-worker timeline samples, 0 = off (MAX_PROFILE_DATA) */
    int32_t result_handles;  /* legacy result-handle table capacity (GTAP_RESULT_HANDLE_CAPACITY) */
    int32_t publish_lazy;    /* 0: publish every task beyond the next batch each round (reference push_batch);
                                1: keep up to 128 ready tasks per queue private until some worker is idle;
                                2: 1 in launches without sort leaves, 0 in the sorting kernel (whose long
                                   rounds leave idle workers waiting for a private reserve) */
    int32_t max_inflight_roots; /* roots admitted but not finished, at most; 0 = no limit */
    int32_t admit_order;     /* GTAP_ADMIT_*: the order in which a batch launch admits its roots */
    int32_t leaf_batch;      /* sort-capable kernel: sort and merge leaves a warp stages in shared memory
                                at once, 1..8, 0 = 1 (one load round trip per batch; each costs 1 KB per
                                warp of shared memory) */
    int32_t join_walk;       /* thread mode, 0..32: in a round of at most this many tasks, the child that
                                completes a built-in fib task's join runs the task's sum at once, and the
                                ancestors' sums whose joins that completes, instead of resuming each in a
                                later round (0 = never).  Each step costs dependent L2 round trips, so full
                                rounds resume as usual; nearly empty rounds (the tree's drain) walk. */
    int32_t sub_rounds;      /* thread mode, 0..8, single queue, launches of fib and n-queens roots only (the
                                kernel without BFS, tree-sum and sort bodies): a round that leaves lanes idle runs up to this
                                many more passes of task bodies on them, each over the newest children the
                                passes before it staged, instead of leaving those children to the next round
                                (0 = one pass).  A tree's ramp-up and drain then go down several levels per
                                round. */
} gtap_config;

/* Admission order of a batch (gtap_launch, gtap_run_host).  Results come back
   in the caller's order whatever the admission order.
   AS_GIVEN:   the roots' order, one persistent launch.
   BY_KIND:    a stable grouping by kind (fib, n-queens, BFS, tree sums, then
               the sorts), one persistent launch: the warps of an SM then run
               one task body at a time instead of all of them at once.
   SPLIT:      BY_KIND, and a thread-mode batch that mixes sorts with other
               kinds runs as two launches back to back on the stream: the
               kernel without sort leaves (more warps per SM, fewer registers)
               over the other kinds, then the sort-capable kernel over the
               sorts.  Block mode admits BY_KIND. */
enum { GTAP_ADMIT_AS_GIVEN = 0, GTAP_ADMIT_BY_KIND = 1, GTAP_ADMIT_SPLIT = 2 };

/* ------------------------------------------------------------------------ */
/* built-in task kinds and root descriptors (NEW)                           */
/* ------------------------------------------------------------------------ */
enum {
    GTAP_KIND_FIB = 1,        /* i0 = n (<= 64), i1 = sequential cutoff (n < i1 runs serially); value = fib(n) */
    GTAP_KIND_NQ = 2,         /* i0 = n (0..32), i1 = cutoff depth (0..255; rows <= i1 fork); value = solutions */
    GTAP_KIND_CILKSORT = 3,   /* p0 = src, p1 = arr (sorted out), p2 = tmp, n = keys, i0 = sort cutoff, i1 = merge cutoff */
    GTAP_KIND_MERGESORT = 4,  /* p0 = src, p1 = arr (sorted out), p2 = tmp, n = keys, i0 = cutoff */
    GTAP_KIND_BFS = 5,        /* p0 = row offsets, p1 = columns, p2 = depth (in/out), i0 = source, i1 = split threshold */
    GTAP_KIND_TREESUM = 6,    /* p0 = left, p1 = right, p2 = value, p3 = subtree sizes, i0 = root node,
                                 i1 = serial cutoff (subtrees of <= i1 nodes are summed serially); value = sum */
    GTAP_KIND_COUNT
};

typedef struct gtap_root {
    int32_t kind;
    int32_t i0, i1, i2;
    int64_t n;
    void* p0;
    void* p1;
    void* p2;
    void* p3;
} gtap_root;

enum { GTAP_ROOT_PENDING = 0, GTAP_ROOT_RUNNING = 1, GTAP_ROOT_DONE = 2 };

typedef struct gtap_root_result {
    int64_t value;          /* fib value, n-queens count, tree sum; 0 for sorts and BFS */
    int64_t tasks;          /* tasks spawned by this root, root included */
    uint64_t t_admit_ns;    /* device %globaltimer when the root task was created */
    uint64_t t_done_ns;     /* device %globaltimer when its last task finished */
    int32_t status;         /* GTAP_ROOT_* */
    int32_t index;
} gtap_root_result;

/* per-worker statistics, summed over workers */
enum {
    GTAP_STAT_TASKS = 0,          /* tasks created */
    GTAP_STAT_EXECUTIONS,         /* task-body executions (incl. resumed continuations) */
    GTAP_STAT_ROUNDS,             /* worker rounds that executed at least one task */
    GTAP_STAT_STEAL_ATTEMPTS,
    GTAP_STAT_STEAL_SUCCESSES,
    GTAP_STAT_STOLEN_TASKS,
    GTAP_STAT_POPS,
    GTAP_STAT_PUBLISHED,          /* tasks made visible to thieves */
    GTAP_STAT_IDLE_POLLS,         /* idle-loop iterations */
    GTAP_STAT_OVERFLOW_PUSHES,
    GTAP_STAT_JOIN_FINISHES,      /* continuations run at their join instead of as a task execution: block mode's
                                     finish-only ones, thread mode's two-result sums (fib) */
    GTAP_STAT_IDLE_NS,            /* nanoseconds workers spent without a task (first failed acquire to the next
                                     success or exit); idle fraction = this / (workers x kernel time) */
    GTAP_STAT_COUNT = 16
};

typedef struct gtap_run_stats {
    uint64_t counters[GTAP_STAT_COUNT];   /* summed over the launches */
    double kernel_ms;        /* CUDA-event time of the persistent launch(es), summed */
    int32_t grid, block, workers;   /* of the sort-capable launch when one ran, else of the last launch */
    int32_t status;
    int32_t launches;        /* persistent worker launches (2 for a split batch, GTAP_ADMIT_SPLIT) */
    int32_t light_workers;   /* workers of the launch without sort leaves, 0 if none ran */
    double light_kernel_ms;  /* part of kernel_ms spent in that launch */
} gtap_run_stats;

#ifdef __cplusplus
}
#endif
#endif /* GTAP_B200_TYPES_H */
