/*
 * gtap.h -- C ABI of the B200 GTaP runtime (libgtap_b200.so).
 *
 * Plain C types only: pointers, sizes and integers.  Every entry point returns
 * an int status: 0 on success, a positive GTAP_ERROR_* runtime code, or a
 * negative value -(cudaError_t) when a CUDA call failed.  Nothing traps.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project root).  Entry points marked NEW have no
 * reference counterpart: they add the multi-root batch and serve modes and
 * the launch-time scheduler parameters that the reference fixes at compile
 * time.
 */
#ifndef GTAP_B200_H
#define GTAP_B200_H

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
    int64_t watchdog_ms;     /* hard wall-clock limit per launch; the kernel returns GTAP_ERROR_TIMEOUT */
    int32_t profile_samples; /* per-worker timeline samples, 0 = off (MAX_PROFILE_DATA) */
    int32_t result_handles;  /* legacy result-handle table capacity (GTAP_RESULT_HANDLE_CAPACITY) */
    int32_t publish_lazy;    /* 0: publish every task beyond the next batch each round (reference push_batch);
                                1: keep up to 128 ready tasks per queue private until some worker is idle */
    int32_t max_inflight_roots; /* roots admitted but not finished, at most; 0 = no limit */
} gtap_config;

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
    GTAP_STAT_COUNT = 16
};

typedef struct gtap_run_stats {
    uint64_t counters[GTAP_STAT_COUNT];
    double kernel_ms;        /* CUDA-event time of the persistent launch */
    int32_t grid, block, workers;
    int32_t status;
} gtap_run_stats;

/* ------------------------------------------------------------------------ */
/* lifecycle -- runtime/detail/thread/gtap_runtime_thread.cuh:338-441       */
/* ------------------------------------------------------------------------ */
/* Fill cfg with defaults for this device (replaces the -D macro defaults). */
int gtap_default_config(gtap_config* cfg);
/* gtap_initialize(): gtap_runtime_thread.cuh:338 -- allocate the arena.  cfg may be NULL. */
int gtap_initialize(const gtap_config* cfg);
/* gtap_finalize(): gtap_runtime_thread.cuh:342 */
int gtap_finalize(void);
/* gtap_reset(): gtap_runtime_thread.cuh:439 -- O(workers) reset, no arena memset. */
int gtap_reset(void);
/* gtap_synchronize(): runtime/detail/common/gtap_runtime_error.cuh:246 */
int gtap_synchronize(void);
/* gtap_get_runtime_error_code(): gtap_runtime_error.cuh:38 */
int gtap_get_runtime_error_code(int* error_code);
/* gtap_check_runtime_error(): gtap_runtime_error.cuh:219 -- prints and returns the device code. */
int gtap_check_runtime_error(void);
/* gtap_get_runtime_error_string(): gtap_runtime_error.cuh:187 */
const char* gtap_get_runtime_error_string(int error_code);
/* Copy of the device error report (gtap_runtime_error.cuh:20-30). NEW accessor. */
int gtap_get_error_report(GtapErrorReport* out);
/* Active configuration (NEW). */
int gtap_get_config(gtap_config* out);

/* ------------------------------------------------------------------------ */
/* launches (NEW; the reference launches exec_kernel<<<GRID,BLOCK>>> with   */
/* one root pushed by __gtap_push_initial_task, gtap_runtime_thread.cuh:818) */
/* ------------------------------------------------------------------------ */
/* Run n_roots roots (device-resident inputs) in ONE persistent launch on the
 * given CUDA stream (NULL = default) and wait for it.  results may be NULL. */
int gtap_launch(const gtap_root* roots, int32_t n_roots, gtap_root_result* results, gtap_run_stats* stats,
                void* stream);
/* The plain per-root baseline: gtap_reset() + one launch per root, as the
 * reference does for repeated runs (gtap_runtime_thread.cuh:349-441). */
int gtap_launch_per_root(const gtap_root* roots, int32_t n_roots, gtap_root_result* results,
                         gtap_run_stats* stats, void* stream);
/* Host-buffer entry point: root pointers refer to HOST memory.  Arrays are
 * copied to the device, the roots run in one launch, and outputs (sorted
 * arrays, BFS depths) are copied back into the same host buffers.
 * h2d_bytes / d2h_bytes (optional) report the bytes moved. */
int gtap_run_host(const gtap_root* roots, int32_t n_roots, gtap_root_result* results, gtap_run_stats* stats,
                  int64_t* h2d_bytes, int64_t* d2h_bytes);

/* Serve mode: a persistent kernel that admits roots while it runs. */
int gtap_serve_start(int32_t ring_capacity, int32_t admit_watermark);
/* Publish n roots (device-resident inputs); returns their indices in *first_index. */
int gtap_serve_enqueue(const gtap_root* roots, int32_t n, int32_t* first_index);
/* Poll completions: writes up to max finished root indices, returns count via *n_out. */
int gtap_serve_poll(int32_t* indices, int32_t max, int32_t* n_out);
/* Read results of finished roots (by index). */
int gtap_serve_results(const int32_t* indices, int32_t n, gtap_root_result* out);
/* Drain outstanding roots, stop the kernel, return its statistics. */
int gtap_serve_shutdown(gtap_run_stats* stats);

/* ------------------------------------------------------------------------ */
/* profiler -- runtime/detail/thread/gtap_profile_thread.cuh:355-358         */
/* ------------------------------------------------------------------------ */
/* Writes ./profile/<app>_warp_*.csv (thread mode) or _block_*.csv (block
 * mode) from the last launch when profile_samples > 0. */
int gtap_visualize_profile(const char* app_name);
/* Same, into a chosen directory (NEW). */
int gtap_write_profile(const char* directory, const char* app_name);

/* ------------------------------------------------------------------------ */
/* seeded workload generators (NEW; stand-ins for gen_vector and SuiteSparse)*/
/* ------------------------------------------------------------------------ */
/* int32 keys = (int32_t)std::mt19937(seed)() */
int gtap_gen_keys(uint32_t seed, int32_t* out, int64_t n);
/* root mix: kind 0 fib / 1 nq / 2 cilksort; see oracle.h for the definition */
int gtap_gen_mix(uint64_t seed, int32_t n_roots, int32_t* kind, int32_t* param, uint64_t* key_seed);
/* R-MAT CSR (a=.57 b=.19 c=.19 d=.05), rows 2^scale+1, cols edge_factor*2^scale */
int gtap_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed, int32_t* row, int32_t* col);
/* random unbalanced binary tree, 48% left split */
int gtap_gen_tree(int32_t n, uint64_t seed, int32_t* left, int32_t* right, int32_t* value, int32_t* size);

/* Exactly-once stress test of the scheduler's deques and overflow queue on the
 * device (NEW, no reference counterpart): every warp publishes unique tokens
 * through the scheduler's own publish path and consumes them by pop, steal
 * and overflow-queue reads.  mode selects the consumers that run while tokens
 * are produced (1 pops, 2 steals, 4 overflow reads; the final drain uses all).
 * Returns 0 when every produced token was consumed exactly once. */
int gtap_selftest_queues(int32_t rounds, int32_t per_round_max, int32_t mode, int64_t* produced,
                         int64_t* consumed, int64_t* duplicates, int64_t* lost);

/* Task-id accounting after the last launch (NEW): out[0] next never-used id,
 * out[1] first id outside the private per-worker ranges, out[2] recycled ids
 * in the pool, out[3] tasks left in the overflow queue, out[4] roots
 * completed, out[5] arena ids, out[6] workers, out[7] status. */
int gtap_get_arena_counters(int64_t* out, int32_t n);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (a serving loop that must avoid an allocation's implicit device-wide
 * synchronisation, or a process whose HBM already belongs to another
 * allocator): runs n_roots roots in one persistent launch with every piece of
 * scheduler scratch in a fixed file-scope device array of about 45 MiB that
 * each GPU loading the library keeps until exit.  d_roots and d_results are
 * device buffers owned by the caller (so are the arrays the roots point to).
 * Needs no gtap_initialize().  Limits: at most 4096 roots (else
 * GTAP_ERROR_INVALID_ARGUMENT), fib / n-queens / BFS / tree-sum kinds only,
 * 2^19 task records shared by live tasks and per-worker free-id caches (a
 * tree that outgrows them fails with GTAP_ERROR_TASK_ID_POOL_LOW_HEADROOM).
 * The first call on a device does a one-time set-up: make it before any
 * stream capture.  Calls share the array: calls that overlap on the GPU race
 * and must be serialised.  Synchronous; returns the device status. */
int gtap_launch_noalloc(const gtap_root* d_roots, int32_t n_roots, gtap_root_result* d_results, void* stream);

/* Library version string (NEW). */
const char* gtap_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GTAP_B200_H */
