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

#include "gtap_types.h"

#ifdef __cplusplus
extern "C" {
#endif

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
/* Run n_roots roots (device-resident inputs) in one persistent launch on the
 * given CUDA stream (NULL = default) and wait for it; under GTAP_ADMIT_SPLIT
 * (the default) a thread-mode batch that mixes sorts with other kinds runs as
 * two launches back to back (gtap_types.h).  results may be NULL; they are
 * returned in the order of roots, results[i].index == i. */
int gtap_launch(const gtap_root* roots, int32_t n_roots, gtap_root_result* results, gtap_run_stats* stats,
                void* stream);
/* The plain per-root baseline: gtap_reset() + one launch per root, as the
 * reference does for repeated runs (gtap_runtime_thread.cuh:349-441). */
int gtap_launch_per_root(const gtap_root* roots, int32_t n_roots, gtap_root_result* results,
                         gtap_run_stats* stats, void* stream);
/* Host-buffer entry point: root pointers refer to HOST memory.  Arrays are
 * copied to the device, the roots run, and outputs (sorted arrays, BFS
 * depths) are copied back into the same host buffers; arrays that continue
 * one another in host memory move in one copy.  Under GTAP_ADMIT_SPLIT a
 * batch of sorts and other kinds runs in three launches: half of the other
 * roots while the sorts' keys are copied in, the sorts, then the other half
 * while the sorted keys are copied out (the copies overlap the launches when
 * the host buffers are pinned).  h2d_bytes / d2h_bytes (optional) report the
 * bytes moved. */
int gtap_run_host(const gtap_root* roots, int32_t n_roots, gtap_root_result* results, gtap_run_stats* stats,
                  int64_t* h2d_bytes, int64_t* d2h_bytes);

/* Serve mode: a persistent kernel that admits roots while it runs. */
int gtap_serve_start(int32_t ring_capacity, int32_t admit_watermark);
/* Publish n roots (device-resident inputs); returns their indices in *first_index. */
int gtap_serve_enqueue(const gtap_root* roots, int32_t n, int32_t* first_index);
/* Poll completions: writes up to max finished root indices, returns count via *n_out. */
int gtap_serve_poll(int32_t* indices, int32_t max, int32_t* n_out);
/* Read results of finished roots by ring slot: during the session, and after
 * gtap_serve_shutdown until the next session or launch. */
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

/* ------------------------------------------------------------------------ */
/* the reference's input files, so its own datasets run when present        */
/* ------------------------------------------------------------------------ */
/* evaluation/util/gen_vector.c:21-60 (save_array / load_array): size_t n, then
 * n int32.  out == NULL: *n_out only.  A file whose size disagrees with n, or
 * capacity < n, is GTAP_ERROR_INVALID_ARGUMENT. */
int gtap_read_array_file(const char* path, int32_t* out, int64_t capacity, int64_t* n_out);
int gtap_write_array_file(const char* path, const int32_t* data, int64_t n);
/* examples/asynchronous_bfs/asynchronous_bfs_thread.cu:69-84 (read_csr_binary):
 * int N, int M, int row[N+1], int col[M].  row == col == NULL: sizes only.
 * Offsets that do not run from 0 to M without decreasing, or a column outside
 * [0, N), are GTAP_ERROR_INVALID_ARGUMENT. */
int gtap_read_csr_file(const char* path, int32_t* row, int64_t row_capacity, int32_t* col, int64_t col_capacity,
                       int32_t* n_out, int32_t* m_out);
int gtap_write_csr_file(const char* path, const int32_t* row, const int32_t* col, int32_t n, int32_t m);

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

/* NEW, a testing aid with no counterpart in the reference.  Moves both cursors
 * of both global rings (the overflow queue and the recycled-id pool) to
 * `position`, leaving them empty, and clears their slots, so that a test
 * reaches the 2^32 wrap of the cursors without 2^32 pushes first.  target 0: the arena of
 * gtap_initialize() (between launches); target 1: the scratch array of
 * gtap_launch_noalloc() on the current device (after its first call). */
int gtap_debug_set_ring_position(int32_t target, uint32_t position);

/* Test aid, host only (no device call): the admission order gtap_launch
 * gives a batch under GTAP_ADMIT_BY_KIND / GTAP_ADMIT_SPLIT.  order[i] = the
 * caller's index of the root admitted i-th (n entries); *n_light = the roots
 * ahead of the first sort (the first launch of a split batch). */
int gtap_debug_admission_order(const gtap_root* roots, int32_t n, int32_t* order, int32_t* n_light);

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
 * stream capture.  Synchronous: returns once the launch has finished, with the
 * device status.  Calls share the array; the library serialises the calls of
 * one process with a lock, and GPU work that bypasses it (another process in
 * the same context) races on the array. */
int gtap_launch_noalloc(const gtap_root* d_roots, int32_t n_roots, gtap_root_result* d_results, void* stream);

/* ------------------------------------------------------------------------ */
/* kernels the caller launches: support for the drop-in task-ABI header     */
/* include/gtap_thread.cuh (NEW).  That header compiles the reference's     */
/* device ABI (runtime/detail/thread/gtap_runtime_thread.cuh:663-1047) into */
/* the caller's exec_kernel and defines the reference's host functions      */
/* (gtap_initialize() etc., returning cudaError_t); these entry points are  */
/* what those functions call, under names that do not collide with them.   */
/* ------------------------------------------------------------------------ */
/* gtap_initialize() of the header (gtap_runtime_thread.cuh:338): allocate the
 * arena for a caller-launched kernel of `workers` warps. */
int gtap_external_initialize(const gtap_config* cfg, int32_t workers);
/* Reset for the next caller launch (gtap_runtime_thread.cuh:349-441
 * __gtap_reset_task_runtime): one root, task id 0, counts as admitted.  Writes
 * the device arena descriptor (arena_bytes must equal its size) that the
 * header copies into its __constant__ symbol. */
int gtap_external_prepare(void* arena_out, int64_t arena_bytes);
/* gtap_finalize() of the header (gtap_runtime_thread.cuh:342). */
int gtap_external_finalize(void);
/* gtap_get_runtime_error_code() of the header (gtap_runtime_error.cuh:38). */
int gtap_external_error_code(int32_t* error_code);
/* gtap_check_runtime_error() of the header (gtap_runtime_error.cuh:219): prints
 * the first device error, returns its code. */
int gtap_external_check(void);

/* Measurement aid (NEW, no reference counterpart): the peak rate, in
 * operations per second, of 32-bit atomic adds to scattered words of an
 * L2-resident 64 MiB table over a full grid -- mode 0 with a return value
 * (atom.add, the join-counter decrement), mode 1 without (red.add).  At least
 * ops (>= 2^20) operations per timed launch.  The denominator of the
 * scheduler's atomic roofline. */
int gtap_measure_atomic_rate(int32_t mode, int64_t ops, double* ops_per_s);

/* Library version string (NEW). */
const char* gtap_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GTAP_B200_H */
