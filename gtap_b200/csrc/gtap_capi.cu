// gtap_capi.cu -- host side of libgtap_b200.so: arena management, launches,
// the plain per-root baseline, host-buffer entry point, serve mode, profiler
// CSVs and the seeded workload generators.  Declarations: include/gtap.h.
//
// Reference host API (paths relative to the reference project root):
//   gtap_initialize / gtap_finalize / gtap_reset   runtime/detail/thread/gtap_runtime_thread.cuh:50-441
//   error report, gtap_synchronize, checks          runtime/detail/common/gtap_runtime_error.cuh:38-249
//   gtap_visualize_profile                          runtime/detail/thread/gtap_profile_thread.cuh:355-358
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <random>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/gtap.h"
#include "gtap_block_programs.cuh"
#include "gtap_programs.cuh"
#include "gtap_selftest.cuh"

using namespace gtap;

namespace {

#define GT_CUDA(call)                                   \
    do {                                                \
        cudaError_t _e = (call);                        \
        if (_e != cudaSuccess) return -(int)_e;         \
    } while (0)

struct Runtime {
    bool initialized = false;
    gtap_config cfg{};
    int device = 0;
    int sm_count = 0;
    int workers = 0;            // arena capacity: max over the kernel variants
    int workers_full = 0;       // thread_worker_kernel<BuiltinProgram>
    int workers_light = 0;      // thread_worker_kernel_lb<BuiltinProgramLight>
    bool fibnq_ok = false;      // thread_worker_kernel_lb<BuiltinProgramFibNq> fits as many workers
    bool stage_light = false;   // g.smem_bytes holds a record stage per warp
    int workers_block = 0;      // block_worker_kernel<BlockProgram>: one worker per block (block mode only)
    int last_workers = 0;       // workers of the last launch
    bool last_block = false;    // the last launch ran the block kernel
    int external_workers = 0;   // workers of a kernel the caller launches (drop-in header), 0 = none
    int warps_per_block = 0;
    size_t smem_bytes = 0;
    size_t smem_full = 0;       // thread_worker_kernel<BuiltinProgram>: smem_bytes + per-warp leaf buffers if they fit
    int leaf_buf = 0;           // leaf input buffers per warp in smem_full

    // arena pieces
    char* records = nullptr;
    void** funcs = nullptr;
    unsigned long long* dq_ctl = nullptr;
    int* dq_slots = nullptr;
    unsigned long long* ring_slots = nullptr;   // overflow ring followed by id pool ring
    unsigned* counters = nullptr;               // small device counters, see kCtr*
    int* hungry = nullptr;                      // kHungryReplicas x kHungryStride
    int* dbg = nullptr;                         // debug builds: 2 x total_ids flags
    unsigned long long* stats = nullptr;
    long long* prof_having = nullptr;
    long long* prof_working = nullptr;
    int* prof_tasks = nullptr;
    gtap_result_handle* handles = nullptr;
    int* handle_meta = nullptr;
    int* staging = nullptr;                     // caller-launched kernels: per-warp staging buffers
    unsigned overflow_log2 = 20, idpool_log2 = 24;

    // roots
    gtap_root* d_roots = nullptr;
    gtap_root_result* d_results = nullptr;
    long long* d_outstanding = nullptr;
    int root_cap = 0;

    // status
    GtapErrorReport* h_report = nullptr;   // mapped pinned
    GtapErrorReport* d_report = nullptr;

    // last launch (profiling)
    bool have_profile = false;

    // serve
    bool serving = false;
    cudaStream_t serve_stream = nullptr;   // runs the persistent kernel
    cudaStream_t feed_stream = nullptr;    // publishes roots while it runs
    unsigned long long* h_done_ring = nullptr;
    unsigned long long* d_done_ring = nullptr;
    unsigned done_cap = 0;
    unsigned serve_published = 0;
    unsigned serve_polled = 0;
    int serve_ring_cap = 0;
    int* h_shutdown_src = nullptr;   // pinned scratch for async copies
    unsigned* h_pub_src = nullptr;
    cudaEvent_t serve_ev0 = nullptr, serve_ev1 = nullptr;
};

// device counter slots inside Runtime::counters
enum {
    kCtrFresh = 0,
    kCtrOvHead,
    kCtrOvTail,
    kCtrPoolHead,
    kCtrPoolTail,
    kCtrNextRoot,
    kCtrCompleted,
    kCtrStatus,
    kCtrAbort,
    kCtrDone,
    kCtrPublished,
    kCtrShutdown,
    kCtrLive,
    kCtrHandleTop,
    kCtrCount = 32
};

Runtime g;
std::mutex g_mu;
char* g_slab = nullptr;      // grow-only device slab for gtap_run_host
size_t g_slab_bytes = 0;

int ilog2_ceil(long long v) {
    int l = 0;
    while ((1ll << l) < v) ++l;
    return l;
}

// Each variant exists for one queue (fewest registers) and for up to kMaxQueues.
const void* kernel_full(int num_queues) {
    return num_queues == 1 ? reinterpret_cast<const void*>(&thread_worker_kernel<BuiltinProgram, 1>)
                           : reinterpret_cast<const void*>(&thread_worker_kernel<BuiltinProgram, kMaxQueues>);
}
const void* kernel_light(int num_queues) {
    return num_queues == 1 ? reinterpret_cast<const void*>(&thread_worker_kernel_lb<BuiltinProgramLight, 1>)
                           : reinterpret_cast<const void*>(&thread_worker_kernel_lb<BuiltinProgramLight, kMaxQueues>);
}
const void* kernel_fibnq(int num_queues) {
    return num_queues == 1 ? reinterpret_cast<const void*>(&thread_worker_kernel_lb<BuiltinProgramFibNq, 1>)
                           : reinterpret_cast<const void*>(&thread_worker_kernel_lb<BuiltinProgramFibNq, kMaxQueues>);
}

// Roots are admitted while at least this many task ids are free (never used
// or recycled).  Ids parked in private ranges and per-warp caches are not
// counted, so the bound stays below half of what is left outside them.
int admission_watermark(int workers) {
    long long outside = g.cfg.total_ids - (long long)workers * g.cfg.ids_per_worker;
    long long w = std::min<long long>(g.cfg.total_ids / 4, outside / 2);
    return (int)std::max<long long>(w, 0);
}

bool roots_need_sorts(const gtap_root* roots, int n) {
    for (int i = 0; i < n; ++i)
        if (roots[i].kind == GTAP_KIND_CILKSORT || roots[i].kind == GTAP_KIND_MERGESORT) return true;
    return false;
}

// layouts the Python binding and other FFI callers mirror
static_assert(sizeof(gtap_config) == 96 && offsetof(gtap_config, admit_order) == 80 &&
                  offsetof(gtap_config, leaf_batch) == 84 && offsetof(gtap_config, join_walk) == 88 &&
                  offsetof(gtap_config, sub_rounds) == 92,
              "gtap_config layout");
static_assert(sizeof(gtap_run_stats) == 168 && offsetof(gtap_run_stats, light_kernel_ms) == 160,
              "gtap_run_stats layout");
static_assert(sizeof(gtap_root) == 56 && sizeof(gtap_root_result) == 40, "root layouts");

bool is_sort_kind(int kind) { return kind == GTAP_KIND_CILKSORT || kind == GTAP_KIND_MERGESORT; }

// Frame bytes the tasks of a root kind use at most: fib, n-queens and BFS
// tasks keep 16-byte frames, so a launch of those alone packs a task record
// (16-byte header + frame) into one 32-byte sector instead of 48 bytes.
static_assert(sizeof(prog::FibFrame) <= 16 && sizeof(prog::NqFrame) <= 16 && sizeof(prog::BfsFrame) <= 16,
              "16-byte frames");
int frame_bytes_of(int kind) {
    return (kind == GTAP_KIND_FIB || kind == GTAP_KIND_NQ || kind == GTAP_KIND_BFS) ? 16 : BuiltinProgram::kFrameBytes;
}

bool only_fib_nq(const gtap_root* roots, int n) {
    for (int i = 0; i < n; ++i)
        if (roots[i].kind != GTAP_KIND_FIB && roots[i].kind != GTAP_KIND_NQ) return false;
    return true;
}

// Record stride of a launch over roots[0, n): the configured one, or less
// when every kind of those roots needs less.
int record_stride_for(const gtap_root* roots, int n) {
    int need = 16;
    for (int i = 0; i < n && need < BuiltinProgram::kFrameBytes; ++i) need = std::max(need, frame_bytes_of(roots[i].kind));
    const int configured = kHdrBytes + ((g.cfg.frame_bytes + 15) / 16) * 16;
    return std::min(configured, kHdrBytes + ((need + 15) / 16) * 16);
}

// Stable grouping of a batch by kind: the kinds without sort leaves first (in
// kind order), then the sorts; kinds out of range lead, so that their error
// is raised before any other root runs.  Fills order (slot -> caller index)
// unless the batch is grouped already, and returns the number of roots ahead
// of the first sort.
int admission_order(const gtap_root* roots, int n, std::vector<int>& order) {
    auto group = [](int kind) {
        if (kind < GTAP_KIND_FIB || kind >= GTAP_KIND_COUNT) return 0;
        return is_sort_kind(kind) ? GTAP_KIND_COUNT + kind : kind;
    };
    constexpr int kGroups = 2 * GTAP_KIND_COUNT;
    int count[kGroups + 1] = {0};
    bool grouped = true;
    int prev = 0;
    for (int i = 0; i < n; ++i) {
        const int k = group(roots[i].kind);
        count[k + 1]++;
        if (k < prev) grouped = false;
        prev = k;
    }
    for (int k = 0; k < kGroups; ++k) count[k + 1] += count[k];
    const int n_light = count[GTAP_KIND_COUNT + 1];
    if (grouped) return n_light;
    order.resize(n);
    for (int i = 0; i < n; ++i) order[count[group(roots[i].kind)]++] = i;
    return n_light;
}

constexpr size_t kBlockSmemBytes = (size_t)BlockProgram::kSmemInts * sizeof(int);

bool block_mode() { return g.cfg.mode == GTAP_MODE_BLOCK; }

// launch the worker kernel variant; A.num_workers must match it.  fibnq:
// the light kernel without the BFS and tree-sum bodies (same occupancy).
cudaError_t launch_worker(const Arena& A, bool light, cudaStream_t s, bool fibnq = false) {
    if (block_mode()) {
        block_worker_kernel<BlockProgram><<<A.num_workers, g.cfg.block, kBlockSmemBytes, s>>>(A);
        return cudaGetLastError();
    }
    const int blocks = A.num_workers / g.warps_per_block;
    const bool one = g.cfg.num_queues == 1;
    if (light && fibnq && g.fibnq_ok) {
        if (one) thread_worker_kernel_lb<BuiltinProgramFibNq, 1><<<blocks, g.cfg.block, g.smem_bytes, s>>>(A);
        else thread_worker_kernel_lb<BuiltinProgramFibNq, kMaxQueues><<<blocks, g.cfg.block, g.smem_bytes, s>>>(A);
        return cudaGetLastError();
    }
    if (light && one) thread_worker_kernel_lb<BuiltinProgramLight, 1><<<blocks, g.cfg.block, g.smem_bytes, s>>>(A);
    else if (light) thread_worker_kernel_lb<BuiltinProgramLight, kMaxQueues><<<blocks, g.cfg.block, g.smem_bytes, s>>>(A);
    else if (one) thread_worker_kernel<BuiltinProgram, 1><<<blocks, g.cfg.block, g.smem_full, s>>>(A);
    else thread_worker_kernel<BuiltinProgram, kMaxQueues><<<blocks, g.cfg.block, g.smem_full, s>>>(A);
    return cudaGetLastError();
}

size_t smem_for(const gtap_config& c) {
    const int wpb = c.block / 32;
    return sizeof(WarpShared) * (size_t)wpb + (size_t)wpb * c.num_queues * (c.spawn_capacity + kLocalCap) * sizeof(int);
}

__global__ void reset_kernel(Arena A, unsigned* counters, int n_roots, int fresh_base) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    const int nctl = A.num_queues * A.num_workers;
    for (int i = tid; i < nctl; i += stride) A.dq_ctl[i] = 0ull;
    const int nst = A.num_workers * GTAP_STAT_COUNT;
    for (int i = tid; i < nst; i += stride) A.stats[i] = 0ull;
    for (int i = tid; i < kHungryReplicas * kHungryStride; i += stride) A.hungry[i] = 0;
    for (int i = tid; i < n_roots; i += stride) {
        A.outstanding[i] = 0;
        gtap_root_result r;
        r.value = 0;
        r.tasks = 0;
        r.t_admit_ns = 0;
        r.t_done_ns = 0;
        r.status = GTAP_ROOT_PENDING;
        r.index = i;
        A.results[i] = r;
    }
    if (tid == 0) {
        counters[kCtrFresh] = (unsigned)fresh_base;
        // the rings keep their positions across launches (slot tags are
        // lap numbers, gtap_ring.h): whatever is still queued is dropped by
        // moving each consumer cursor to its producer cursor
        counters[kCtrOvHead] = counters[kCtrOvTail];
        counters[kCtrPoolHead] = counters[kCtrPoolTail];
        counters[kCtrNextRoot] = 0;
        counters[kCtrCompleted] = 0;
        counters[kCtrStatus] = 0;
        counters[kCtrAbort] = 0;
        counters[kCtrDone] = 0;
        counters[kCtrPublished] = 0;
        counters[kCtrShutdown] = 0;
        counters[kCtrLive] = 0;
        counters[kCtrHandleTop] = 0;
    }
}

// first_root: the batch's roots, results and balances start at this slot
Arena make_arena(int n_roots, int mode, int workers, int first_root = 0) {
    Arena A{};
    const gtap_config& c = g.cfg;
    A.num_workers = workers;
    A.warps_per_block = g.warps_per_block;
    A.num_queues = c.num_queues;
    A.deque_cap_log2 = ilog2_ceil(c.deque_capacity);
    A.steal_batch = c.steal_batch;
    A.victim_policy = c.victim_policy;
    A.probe_width = c.probe_width;
    A.spawn_cap = c.spawn_capacity;
    A.ids_per_worker = c.ids_per_worker;
    A.avail_target = kAvailCap - 32;
    A.rec_stride = kHdrBytes + ((c.frame_bytes + 15) / 16) * 16;
    A.admit_batch = c.admit_batch;
    A.mode = mode;
    A.publish_lazy = c.publish_lazy != 0 ? 1 : 0;
    A.join_walk = c.join_walk;
    A.sub_rounds = c.sub_rounds;
    A.max_inflight = c.max_inflight_roots;
    A.total_ids = (int)c.total_ids;
    A.watchdog_ns = (unsigned long long)c.watchdog_ms * 1000000ull;
    A.records = g.records;
    A.funcs = g.funcs;
    A.dq_ctl = g.dq_ctl;
    A.dq_slots = g.dq_slots;
    A.overflow.slots = g.ring_slots;
    A.overflow.head = g.counters + kCtrOvHead;
    A.overflow.tail = g.counters + kCtrOvTail;
    A.overflow.cap_log2 = g.overflow_log2;
    A.idpool.slots = g.ring_slots + (1ull << g.overflow_log2);
    A.idpool.head = g.counters + kCtrPoolHead;
    A.idpool.tail = g.counters + kCtrPoolTail;
    A.idpool.cap_log2 = g.idpool_log2;
    A.fresh_next = g.counters + kCtrFresh;
    A.roots = g.d_roots + first_root;
    A.results = g.d_results + first_root;
    A.outstanding = g.d_outstanding + first_root;
    A.n_roots = n_roots;
    A.next_root = g.counters + kCtrNextRoot;
    A.published = g.counters + kCtrPublished;
    A.shutdown = reinterpret_cast<const int*>(g.counters + kCtrShutdown);
    A.completed = g.counters + kCtrCompleted;
    A.done_ring = g.d_done_ring;
    A.done_ring_cap = g.done_cap;
    A.live_tasks = reinterpret_cast<int*>(g.counters + kCtrLive);
    A.admit_watermark = 0;
    A.status = reinterpret_cast<int*>(g.counters + kCtrStatus);
    A.abort_flag = reinterpret_cast<int*>(g.counters + kCtrAbort);
    A.done_flag = reinterpret_cast<int*>(g.counters + kCtrDone);
    A.report = g.d_report;
    A.stats = g.stats;
    A.hungry = g.hungry;
    A.dbg_live = g.dbg;
    A.dbg_exec = g.dbg ? g.dbg + c.total_ids : nullptr;
    A.dbg_slotpos = g.dbg ? reinterpret_cast<unsigned*>(g.dbg + 2 * c.total_ids) : nullptr;
    A.prof_having = g.prof_having;
    A.prof_working = g.prof_working;
    A.prof_tasks = g.prof_tasks;
    A.prof_cap = c.profile_samples;
    A.handles = g.handles;
    A.handle_top = reinterpret_cast<int*>(g.counters + kCtrHandleTop);
    A.handle_meta = g.handle_meta;
    A.handle_cap = c.result_handles;
    A.staging = g.staging;
    A.leaf_buf = g.leaf_buf;
    // the kernels this arena launches hold a record stage per warp (the light
    // kernels in g.smem_bytes, the sorting kernel in its leaf buffers)
    A.rec_prefetch = g.stage_light ? 1 : 0;
    return A;
}

int ensure_root_capacity(int n) {
    if (n <= g.root_cap) return 0;
    int cap = std::max(n, std::max(1024, g.root_cap * 2));
    if (g.d_roots) cudaFree(g.d_roots);
    if (g.d_results) cudaFree(g.d_results);
    if (g.d_outstanding) cudaFree(g.d_outstanding);
    g.d_roots = nullptr;
    g.d_results = nullptr;
    g.d_outstanding = nullptr;
    g.root_cap = 0;
    GT_CUDA(cudaMalloc(&g.d_roots, sizeof(gtap_root) * cap));
    GT_CUDA(cudaMalloc(&g.d_results, sizeof(gtap_root_result) * cap));
    GT_CUDA(cudaMalloc(&g.d_outstanding, sizeof(long long) * cap));
    g.root_cap = cap;
    return 0;
}

int validate_config(const gtap_config& c) {
    if (c.mode != GTAP_MODE_THREAD && c.mode != GTAP_MODE_BLOCK) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.block <= 0 || c.block % 32 != 0 || c.block > 1024) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.grid < 0) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.num_queues < 1 || c.num_queues > kMaxQueues) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.deque_capacity < 64 || c.deque_capacity > (1 << 20) || (c.deque_capacity & (c.deque_capacity - 1)))
        return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.steal_batch < 1 || c.steal_batch > 32) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.probe_width < 1 || c.probe_width > 32) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.victim_policy < 0 || c.victim_policy > 2) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.spawn_capacity < 64 || c.spawn_capacity > 8192) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.ids_per_worker < 64) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.total_ids < 128 || c.total_ids > (1ll << kIdBits)) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.frame_bytes < 16 || c.frame_bytes > 4096) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.admit_batch < 1 || c.admit_batch > 32) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.watchdog_ms < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.profile_samples < 0 || c.result_handles < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.publish_lazy < 0 || c.publish_lazy > 2 || c.max_inflight_roots < 0) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.admit_order < GTAP_ADMIT_AS_GIVEN || c.admit_order > GTAP_ADMIT_SPLIT) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.leaf_batch < 0 || c.leaf_batch > 8) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.join_walk < 0 || c.join_walk > 32) return GTAP_ERROR_INVALID_ARGUMENT;
    if (c.sub_rounds < 0 || c.sub_rounds > 8) return GTAP_ERROR_INVALID_ARGUMENT;
    return 0;
}

void free_all() {
    auto F = [](auto*& p) {
        if (p) cudaFree((void*)p);
        p = nullptr;
    };
    F(g.records);
    F(g.funcs);
    F(g.dq_ctl);
    F(g.dq_slots);
    F(g.ring_slots);
    F(g.counters);
    F(g.hungry);
    F(g.dbg);
    F(g.stats);
    F(g.prof_having);
    F(g.prof_working);
    F(g.prof_tasks);
    F(g.handles);
    F(g.handle_meta);
    F(g.staging);
    F(g.d_roots);
    F(g.d_results);
    F(g.d_outstanding);
    g.root_cap = 0;
    if (g.h_report) cudaFreeHost(g.h_report);
    g.h_report = nullptr;
    if (g_slab) cudaFree(g_slab);
    g_slab = nullptr;
    g_slab_bytes = 0;
    g.d_report = nullptr;
    g.initialized = false;
    g.external_workers = 0;
}

int read_status() {
    int st = 0;
    cudaError_t e = cudaMemcpy(&st, g.counters + kCtrStatus, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return -(int)e;
    return st;
}

int collect_stats(gtap_run_stats* stats) {
    if (!stats) return 0;
    const int W = g.last_workers;
    std::vector<unsigned long long> h((size_t)W * GTAP_STAT_COUNT);
    GT_CUDA(cudaMemcpy(h.data(), g.stats, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (int i = 0; i < GTAP_STAT_COUNT; ++i) stats->counters[i] = 0;
    for (int w = 0; w < W; ++w)
        for (int i = 0; i < GTAP_STAT_COUNT; ++i) stats->counters[i] += h[(size_t)w * GTAP_STAT_COUNT + i];
    stats->grid = g.last_block ? W : W / g.warps_per_block;
    stats->block = g.cfg.block;
    stats->workers = W;
    return 0;
}

// One persistent launch over the roots already in g.d_roots[first_root, first_root + n_roots).
// rec_stride > 0: the record stride of this launch (at most the configured one).
int launch_resident(int n_roots, cudaStream_t s, float* ms_out, bool light, int first_root = 0, int rec_stride = 0,
                    bool fibnq = false) {
    if (g.cfg.profile_samples > 0) {
        size_t n = (size_t)g.workers * g.cfg.profile_samples;
        GT_CUDA(cudaMemsetAsync(g.prof_having, 0, n * sizeof(long long), s));
        GT_CUDA(cudaMemsetAsync(g.prof_working, 0, n * sizeof(long long), s));
        GT_CUDA(cudaMemsetAsync(g.prof_tasks, 0, n * sizeof(int), s));
    }
#ifdef GTAP_DEBUG_IDS
    GT_CUDA(cudaMemsetAsync(g.dbg, 0, (size_t)2 * g.cfg.total_ids * sizeof(int), s));
    GT_CUDA(cudaMemsetAsync(g.dbg + 2 * g.cfg.total_ids, 0xFF,
                            (size_t)g.cfg.num_queues * g.workers * g.cfg.deque_capacity * sizeof(int), s));
#endif
    const int W = block_mode() ? g.workers_block : light ? g.workers_light : g.workers_full;
    g.last_workers = W;
    g.last_block = block_mode();
    Arena A = make_arena(n_roots, 0, W, first_root);
    if (rec_stride > 0 && rec_stride < A.rec_stride) A.rec_stride = rec_stride;
    if (!light && !block_mode()) {
        A.rec_prefetch = g.leaf_buf > 0 ? 1 : 0;   // the sorting kernel: its leaf buffers
        if (g.cfg.publish_lazy == 2) A.publish_lazy = 0;
    }
    const int fresh_base = W * g.cfg.ids_per_worker;
    A.admit_watermark = admission_watermark(W);
    reset_kernel<<<std::max(1, std::min(1184, (std::max(n_roots, W * g.cfg.num_queues) + 255) / 256)), 256, 0,
                   s>>>(A, g.counters, n_roots, fresh_base);
    GT_CUDA(cudaGetLastError());
    cudaEvent_t e0, e1;
    GT_CUDA(cudaEventCreate(&e0));
    GT_CUDA(cudaEventCreate(&e1));
    GT_CUDA(cudaEventRecord(e0, s));
    cudaError_t le = launch_worker(A, light, s, fibnq);
    GT_CUDA(cudaEventRecord(e1, s));
    cudaError_t se = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (le != cudaSuccess) return -(int)le;
    if (se != cudaSuccess) return -(int)se;
    if (ms_out) *ms_out = ms;
    g.have_profile = g.cfg.profile_samples > 0;
    return read_status();
}

// The one root of a kernel the caller launches (drop-in header): task id 0,
// created on the device by __gtap_push_initial_task, counts as admitted.
__global__ void external_root_kernel(Arena A, unsigned* counters) {
    A.outstanding[0] = 1;
    gtap_root_result r;
    r.value = 0;
    r.tasks = 1;
    r.t_admit_ns = global_ns();
    r.t_done_ns = 0;
    r.status = GTAP_ROOT_RUNNING;
    r.index = 0;
    A.results[0] = r;
    counters[kCtrNextRoot] = 1;   // nothing left to admit
}


// Hooks of a host-buffer batch (gtap_run_host): the sort roots' inputs arrive
// on another stream while a launch without sorts runs, and their outputs leave
// while the last launch runs.
struct BatchHooks {
    std::function<int()> before_launches;   // issues the input copies, after the root table's copy
    cudaEvent_t sort_inputs = nullptr;   // recorded after the sort roots' input copies
    std::function<int()> after_sorts;    // issues the sort roots' output copies
    bool halve_light = false;            // the other roots in two launches of alternate roots, one on
                                         // each side of the sorts
};

// A batch launch (the caller holds g_mu and has checked the arguments): the
// roots in admission order in g.d_roots, one launch or a split into
// segments, results back in the caller's order.
int run_batch(const gtap_root* roots, int n_roots, gtap_root_result* results, gtap_run_stats* stats,
              cudaStream_t s, const BatchHooks* hooks) {
    if (g.h_report) memset(g.h_report, 0, sizeof(GtapErrorReport));
    int rc = ensure_root_capacity(n_roots);
    if (rc) return rc;
    const bool sorts = roots_need_sorts(roots, n_roots);
    if (!block_mode() && sorts && g.workers_full == 0) return GTAP_ERROR_INVALID_ARGUMENT;

    // admission order: slot i of the device table holds the caller's root order[i]
    std::vector<int> order;
    int n_light = sorts ? 0 : n_roots;
    if (g.cfg.admit_order != GTAP_ADMIT_AS_GIVEN) n_light = admission_order(roots, n_roots, order);
    const bool split = !block_mode() && g.cfg.admit_order == GTAP_ADMIT_SPLIT && g.cfg.profile_samples == 0 &&
                       n_light > 0 && n_light < n_roots;
    const bool halves = split && hooks && hooks->halve_light && n_light >= 2;
    if (halves) {
        // two launches of about equal work: alternate roots of the grouped
        // order, so that each half keeps the grouping and gets half of each kind
        if (order.empty()) {
            order.resize(n_roots);
            for (int i = 0; i < n_roots; ++i) order[i] = i;
        }
        std::vector<int> light(order.begin(), order.begin() + n_light);
        int w = 0;
        for (int i = 0; i < n_light; i += 2) order[w++] = light[i];
        for (int i = 1; i < n_light; i += 2) order[w++] = light[i];
    }
    const gtap_root* table = roots;
    std::vector<gtap_root> permuted;
    if (!order.empty()) {
        permuted.resize(n_roots);
        for (int i = 0; i < n_roots; ++i) permuted[i] = roots[order[i]];
        table = permuted.data();
    }
    GT_CUDA(cudaMemcpyAsync(g.d_roots, table, sizeof(gtap_root) * n_roots, cudaMemcpyHostToDevice, s));
    // the inputs' copies queue behind the root table on the copy engine, so
    // that a long one does not hold up the first launch
    if (hooks && hooks->before_launches) {
        int hc = hooks->before_launches();
        if (hc) return hc;
    }

    // segments: one launch, or (split) the kernel without sort leaves over
    // slots [0, n_light) and the sort-capable kernel over [n_light, n_roots)
    struct Segment {
        int first, count;
        bool light;
    };
    std::vector<Segment> segs;
    if (!split) {
        segs.push_back({0, n_roots, !sorts});
    } else if (halves) {
        const int a = (n_light + 1) / 2;
        segs.push_back({0, a, true});
        segs.push_back({n_light, n_roots - n_light, false});
        segs.push_back({a, n_light - a, true});
    } else {
        segs.push_back({0, n_light, true});
        segs.push_back({n_light, n_roots - n_light, false});
    }

    double ms_total = 0, ms_light = 0;
    int st = 0, launches = 0, light_workers = 0;
    std::vector<char> ran(n_roots, 0);
    gtap_run_stats acc{}, shape{};
    bool have_shape = false;
    for (const Segment& sg : segs) {
        const bool needs_sorts = !sg.light || block_mode();
        if (needs_sorts && hooks && hooks->sort_inputs) GT_CUDA(cudaStreamWaitEvent(s, hooks->sort_inputs, 0));
        float ms = 0.f;
        const int stride = block_mode() ? 0 : record_stride_for(table + sg.first, sg.count);
        st = launch_resident(sg.count, s, &ms, sg.light && !block_mode(), sg.first, stride,
                             only_fib_nq(table + sg.first, sg.count));
        ++launches;
        ms_total += ms;
        for (int i = sg.first; i < sg.first + sg.count; ++i) ran[i] = 1;
        if (sg.light && !block_mode()) {
            ms_light += ms;
            light_workers = g.last_workers;
        }
        if (stats) {
            gtap_run_stats one{};
            int cs = collect_stats(&one);
            if (cs) return cs;
            for (int k = 0; k < GTAP_STAT_COUNT; ++k) acc.counters[k] += one.counters[k];
            if (!have_shape || !sg.light) shape = one;   // the sort-capable launch's shape, if one ran
            have_shape = true;
        }
        if (st != 0) break;
        if (!sg.light && hooks && hooks->after_sorts) {
            st = hooks->after_sorts();
            if (st != 0) break;
        }
    }

    if (results) {
        gtap_root_result* dst = results;
        std::vector<gtap_root_result> staged;
        if (!order.empty()) {
            staged.resize(n_roots);
            dst = staged.data();
        }
        GT_CUDA(cudaMemcpyAsync(dst, g.d_results, sizeof(gtap_root_result) * n_roots, cudaMemcpyDeviceToHost, s));
        GT_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < n_roots; ++i) {
            if (!ran[i]) {   // a segment after a failed launch: never admitted
                dst[i] = gtap_root_result{};
                dst[i].status = GTAP_ROOT_PENDING;
            }
            const int caller = order.empty() ? i : order[i];
            dst[i].index = caller;
            if (!order.empty()) results[caller] = dst[i];
        }
    }
    if (stats) {
        *stats = shape;
        for (int k = 0; k < GTAP_STAT_COUNT; ++k) stats->counters[k] = acc.counters[k];
        stats->kernel_ms = ms_total;
        stats->status = st;
        stats->launches = launches;
        stats->light_workers = light_workers;
        stats->light_kernel_ms = ms_light;
    }
    return st;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

#ifdef GTAP_DEBUG_IDS
const char* gtap_version(void) { return "gtap_b200 0.1 (sm_100a, id checks)"; }
#else
const char* gtap_version(void) { return "gtap_b200 0.1 (sm_100a)"; }
#endif

int gtap_default_config(gtap_config* cfg) {
    if (!cfg) return GTAP_ERROR_INVALID_ARGUMENT;
    memset(cfg, 0, sizeof(*cfg));
    cfg->mode = GTAP_MODE_THREAD;
    cfg->grid = 0;
    cfg->block = 256;
    cfg->num_queues = 1;
    cfg->deque_capacity = 4096;
    cfg->steal_batch = 32;
    cfg->victim_policy = GTAP_VICTIM_PROBE_MAX;
    cfg->probe_width = 16;
    cfg->spawn_capacity = 512;
    cfg->ids_per_worker = 1024;
    cfg->total_ids = 1 << 26;
    cfg->frame_bytes = BuiltinProgram::kFrameBytes;
    cfg->admit_batch = 1;
    cfg->watchdog_ms = 20000;
    cfg->profile_samples = 0;
    cfg->result_handles = 1000;
    cfg->publish_lazy = 0;
    cfg->max_inflight_roots = 0;
    cfg->admit_order = GTAP_ADMIT_SPLIT;
    cfg->leaf_batch = 1;
    cfg->join_walk = 0;
    cfg->sub_rounds = 0;
    return 0;
}

// external_workers > 0: the arena also serves a kernel the caller launches
// with that many warps (the drop-in task-ABI header's exec_kernel).
static int initialize_impl(const gtap_config* cfg_in, int external_workers) {
    if (g.serving) return GTAP_ERROR_BUSY;
    if (g.initialized) free_all();
    gtap_config c;
    if (cfg_in) c = *cfg_in;
    else gtap_default_config(&c);
    int v = validate_config(c);
    if (v) return v;
    GT_CUDA(cudaGetDevice(&g.device));
    GT_CUDA(cudaDeviceGetAttribute(&g.sm_count, cudaDevAttrMultiProcessorCount, g.device));
    const size_t smem = smem_for(c);
    int smem_optin = 0;
    GT_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, g.device));
    // the light kernels also hold a record stage per warp (16 bytes of slack
    // to align it), when the block's shared memory can hold it
    size_t smem_light = smem + (size_t)(c.block / 32) * (kRecStageBytes + 16);
    const bool stage_light = smem_light <= (size_t)smem_optin;
    if (!stage_light) smem_light = smem;
    // the sorting kernel also holds leaf buffers: per warp leaf_batch input
    // buffers and an output buffer, or fewer inputs when the block's shared
    // memory cannot hold them
    int leaf_buf = c.leaf_batch > 0 ? c.leaf_batch : 1;
    size_t smem_full = smem;
    for (; leaf_buf > 0; leaf_buf /= 2) {
        smem_full = smem + (size_t)(c.block / 32) * (leaf_buf + 1) * BuiltinProgram::kLeafKeys * sizeof(int);
        if (smem_full <= (size_t)smem_optin) break;
    }
    if (leaf_buf == 0) smem_full = smem;
    int per_sm_full = 0, per_sm_light = 0;
    GT_CUDA(cudaFuncSetAttribute(kernel_full(c.num_queues), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_full));
    GT_CUDA(cudaFuncSetAttribute(kernel_light(c.num_queues), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_light));
    if (c.block <= kFullKernelThreads)   // the sorting kernel's launch bound
        GT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_full, kernel_full(c.num_queues), c.block, smem_full));
    GT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_light, kernel_light(c.num_queues), c.block, smem_light));
    if (per_sm_light < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    {
        int per_sm_fibnq = 0;
        GT_CUDA(cudaFuncSetAttribute(kernel_fibnq(c.num_queues), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_light));
        GT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_fibnq, kernel_fibnq(c.num_queues), c.block,
                                                              smem_light));
        g.fibnq_ok = per_sm_fibnq >= per_sm_light;
    }
    // one resident wave per variant; grid = 0 fills the GPU, otherwise cap it
    auto pick = [&](int per_sm) {
        int cap = per_sm * g.sm_count;
        return c.grid == 0 ? cap : std::min(c.grid, cap);
    };
    const int grid_light = pick(per_sm_light);
    const int grid_full = per_sm_full > 0 ? pick(per_sm_full) : 0;
    g.warps_per_block = c.block / 32;
    g.workers_light = grid_light * g.warps_per_block;
    g.workers_full = grid_full * g.warps_per_block;
    g.workers_block = 0;
    if (c.mode == GTAP_MODE_BLOCK) {
        // one worker per block; the grid fills the GPU unless capped
        if (c.block > kBMaxThreads) return GTAP_ERROR_INVALID_ARGUMENT;
        int per_sm_block = 0;
        GT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_block, &block_worker_kernel<BlockProgram>, c.block,
                                                              kBlockSmemBytes));
        if (per_sm_block < 1) return GTAP_ERROR_INVALID_ARGUMENT;
        g.workers_block = pick(per_sm_block);
    }
    g.workers = std::max(std::max(std::max(g.workers_light, g.workers_full), external_workers), g.workers_block);
    g.external_workers = external_workers;
    g.last_workers = g.workers_light;
    if (c.grid == 0) c.grid = c.mode == GTAP_MODE_BLOCK ? g.workers_block : std::max(grid_light, grid_full);
    if ((long long)g.workers * c.ids_per_worker + 1 > c.total_ids) {
        // private ranges that would not fit may use at most half of the arena
        // (id 0 may be reserved for a caller-launched kernel's initial task)
        c.ids_per_worker = (int)((c.total_ids / 2 - 1) / g.workers);
        if (c.ids_per_worker < 64) return GTAP_ERROR_INVALID_ARGUMENT;
    }
    g.cfg = c;
    g.smem_bytes = smem_light;
    g.stage_light = stage_light;
    g.smem_full = smem_full;
    g.leaf_buf = leaf_buf;

    const int stride = kHdrBytes + ((c.frame_bytes + 15) / 16) * 16;
    GT_CUDA(cudaMalloc(&g.records, (size_t)(c.total_ids + 1) * stride));   // + spare record for failed allocations
    GT_CUDA(cudaMalloc(&g.funcs, (size_t)c.total_ids * sizeof(void*)));
    GT_CUDA(cudaMalloc(&g.dq_ctl, (size_t)c.num_queues * g.workers * sizeof(unsigned long long)));
    GT_CUDA(cudaMalloc(&g.dq_slots, (size_t)c.num_queues * g.workers * c.deque_capacity * sizeof(int)));
    // both rings hold every id of the arena, so neither can overrun
    g.idpool_log2 = (unsigned)ilog2_ceil(c.total_ids + 1);
    g.overflow_log2 = g.idpool_log2;
    size_t nslots = (1ull << g.overflow_log2) + (1ull << g.idpool_log2);
    GT_CUDA(cudaMalloc(&g.ring_slots, nslots * sizeof(unsigned long long)));
    GT_CUDA(cudaMemset(g.ring_slots, 0, nslots * sizeof(unsigned long long)));
    GT_CUDA(cudaMalloc(&g.counters, kCtrCount * sizeof(unsigned)));
    GT_CUDA(cudaMemset(g.counters, 0, kCtrCount * sizeof(unsigned)));
    GT_CUDA(cudaMalloc(&g.hungry, kHungryReplicas * kHungryStride * sizeof(int)));
    GT_CUDA(cudaMemset(g.hungry, 0, kHungryReplicas * kHungryStride * sizeof(int)));
#ifdef GTAP_DEBUG_IDS
    GT_CUDA(cudaMalloc(&g.dbg, ((size_t)2 * c.total_ids + (size_t)c.num_queues * g.workers * c.deque_capacity) * sizeof(int)));
#endif
    GT_CUDA(cudaMalloc(&g.stats, (size_t)g.workers * GTAP_STAT_COUNT * sizeof(unsigned long long)));
    if (c.profile_samples > 0) {
        size_t n = (size_t)g.workers * c.profile_samples;
        GT_CUDA(cudaMalloc(&g.prof_having, n * sizeof(long long)));
        GT_CUDA(cudaMalloc(&g.prof_working, n * sizeof(long long)));
        GT_CUDA(cudaMalloc(&g.prof_tasks, n * sizeof(int)));
    }
    GT_CUDA(cudaMalloc(&g.handles, (size_t)c.result_handles * sizeof(gtap_result_handle)));
    GT_CUDA(cudaMalloc(&g.handle_meta, (size_t)c.total_ids * 3 * sizeof(int)));
    if (external_workers > 0)
        GT_CUDA(cudaMalloc(&g.staging, (size_t)external_workers * c.num_queues * (c.spawn_capacity + kLocalCap) * sizeof(int)));
    GT_CUDA(cudaHostAlloc(&g.h_report, sizeof(GtapErrorReport), cudaHostAllocMapped));
    memset(g.h_report, 0, sizeof(GtapErrorReport));
    GT_CUDA(cudaHostGetDevicePointer(&g.d_report, g.h_report, 0));
    int rc = ensure_root_capacity(4096);
    if (rc) return rc;
    g.initialized = true;
    GT_CUDA(cudaDeviceSynchronize());
    return 0;
}

int gtap_initialize(const gtap_config* cfg_in) {
    std::lock_guard<std::mutex> lk(g_mu);
    return initialize_impl(cfg_in, 0);
}

int gtap_finalize(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.serving) return GTAP_ERROR_BUSY;
    if (!g.initialized) return 0;
    cudaDeviceSynchronize();
    free_all();
    return 0;
}

int gtap_reset(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.serving) return GTAP_ERROR_BUSY;
    if (g.h_report) memset(g.h_report, 0, sizeof(GtapErrorReport));
    Arena A = make_arena(0, 0, g.workers);
    reset_kernel<<<64, 256>>>(A, g.counters, 0, g.workers * g.cfg.ids_per_worker);
    GT_CUDA(cudaGetLastError());
    GT_CUDA(cudaDeviceSynchronize());
    return 0;
}

int gtap_external_initialize(const gtap_config* cfg, int32_t workers) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (workers < 1 || !cfg) return GTAP_ERROR_INVALID_ARGUMENT;
    if (g.serving) return GTAP_ERROR_BUSY;
    if (g.initialized) free_all();
    return initialize_impl(cfg, workers);
}

int gtap_external_prepare(void* arena_out, int64_t arena_bytes) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized || g.external_workers == 0) return GTAP_ERROR_NOT_INITIALIZED;
    if (!arena_out || arena_bytes != (int64_t)sizeof(Arena)) return GTAP_ERROR_INVALID_ARGUMENT;
    if (g.serving) return GTAP_ERROR_BUSY;
    if (g.h_report) memset(g.h_report, 0, sizeof(GtapErrorReport));
    if (g.cfg.profile_samples > 0) {
        size_t n = (size_t)g.workers * g.cfg.profile_samples;
        GT_CUDA(cudaMemset(g.prof_having, 0, n * sizeof(long long)));
        GT_CUDA(cudaMemset(g.prof_working, 0, n * sizeof(long long)));
        GT_CUDA(cudaMemset(g.prof_tasks, 0, n * sizeof(int)));
    }
    const int W = g.external_workers;
    g.last_workers = W;
    g.last_block = false;
    Arena A = make_arena(1, 0, W);
    A.id_base = 1;   // id 0 is the initial task's (its frame is __gtap_get_task_data(0))
    A.admit_watermark = 0;
    reset_kernel<<<64, 256>>>(A, g.counters, 1, 1 + W * g.cfg.ids_per_worker);
    GT_CUDA(cudaGetLastError());
    external_root_kernel<<<1, 1>>>(A, g.counters);
    GT_CUDA(cudaGetLastError());
    GT_CUDA(cudaDeviceSynchronize());
    g.have_profile = g.cfg.profile_samples > 0;
    memcpy(arena_out, &A, sizeof(Arena));
    return 0;
}

int gtap_external_finalize(void) { return gtap_finalize(); }

int gtap_external_error_code(int32_t* error_code) { return gtap_get_runtime_error_code(error_code); }

int gtap_external_check(void) { return gtap_check_runtime_error(); }

int gtap_get_config(gtap_config* out) {
    if (!out) return GTAP_ERROR_INVALID_ARGUMENT;
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    *out = g.cfg;
    return 0;
}

const char* gtap_get_runtime_error_string(int code) {
    static const char* const msg[GTAP_ERROR_COUNT] = {
        "No error",
        "Invalid queue index",
        "Invalid queue index after join",
        "Queue overflow",
        "Result handle table overflow",
        "Task ID pool exhausted",
        "Task ID pool exhausted",
        "Generated task ID buffer overflow",
        "Invalid taskwait lowering",
        "Timeout",
        "Invalid task kind",
        "Invalid argument",
        "Runtime not initialized",
        "Runtime busy",
    };
    if (code >= 0 && code < GTAP_ERROR_COUNT) return msg[code];
    if (code < 0) return cudaGetErrorString((cudaError_t)(-code));
    return "Unknown error";
}

int gtap_get_runtime_error_code(int* error_code) {
    if (!error_code) return GTAP_ERROR_INVALID_ARGUMENT;
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    int st = read_status();
    if (st < 0) return st;
    *error_code = st;
    return 0;
}

int gtap_get_error_report(GtapErrorReport* out) {
    if (!out) return GTAP_ERROR_INVALID_ARGUMENT;
    if (!g.initialized || !g.h_report) return GTAP_ERROR_NOT_INITIALIZED;
    *out = *g.h_report;
    return 0;
}

int gtap_check_runtime_error(void) {
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.h_report && g.h_report->valid) {
        const GtapErrorReport* r = g.h_report;
        printf("GTaP Runtime Error at block %d, thread %d: %s (code=%d, tid=%d, queue=%d, value=%d, limit=%d) (source_line: %d)\n",
               r->block_idx, r->thread_idx, gtap_get_runtime_error_string(r->code), r->code, r->tid, r->queue_idx,
               r->value, r->limit, r->src_line);
        return r->code;
    }
    int st = read_status();
    if (st > 0) printf("GTaP Runtime Error: %s (code: %d)\n", gtap_get_runtime_error_string(st), st);
    return st;
}

int gtap_synchronize(void) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        printf("CUDA ERROR: %s\n", cudaGetErrorString(e));
        return -(int)e;
    }
    if (!g.initialized) return 0;
    return gtap_check_runtime_error();
}

int gtap_launch(const gtap_root* roots, int32_t n_roots, gtap_root_result* results, gtap_run_stats* stats,
                void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.serving) return GTAP_ERROR_BUSY;
    if (!roots || n_roots < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    return run_batch(roots, n_roots, results, stats, reinterpret_cast<cudaStream_t>(stream), nullptr);
}

int gtap_launch_per_root(const gtap_root* roots, int32_t n_roots, gtap_root_result* results,
                         gtap_run_stats* stats, void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.serving) return GTAP_ERROR_BUSY;
    if (!roots || n_roots < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    int rc = ensure_root_capacity(1);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    gtap_run_stats total{};
    double ms_total = 0, ms_light = 0;
    int st = 0, launches = 0, light_workers = 0;
    for (int i = 0; i < n_roots && st == 0; ++i) {
        GT_CUDA(cudaMemcpyAsync(g.d_roots, roots + i, sizeof(gtap_root), cudaMemcpyHostToDevice, s));
        float ms = 0.f;
        const bool light = !roots_need_sorts(roots + i, 1);
        if (!block_mode() && !light && g.workers_full == 0) return GTAP_ERROR_INVALID_ARGUMENT;
        st = launch_resident(1, s, &ms, light);
        ms_total += ms;
        ++launches;
        if (light && !block_mode()) {
            ms_light += ms;
            light_workers = g.last_workers;
        }
        if (results) {
            GT_CUDA(cudaMemcpyAsync(results + i, g.d_results, sizeof(gtap_root_result), cudaMemcpyDeviceToHost, s));
        }
        if (stats) {
            gtap_run_stats one{};
            int cs = collect_stats(&one);
            if (cs) return cs;
            for (int k = 0; k < GTAP_STAT_COUNT; ++k) total.counters[k] += one.counters[k];
        }
    }
    GT_CUDA(cudaStreamSynchronize(s));
    if (results)
        for (int i = 0; i < n_roots; ++i) results[i].index = i;
    if (stats) {
        *stats = total;
        stats->kernel_ms = ms_total;
        stats->grid = g.last_block ? g.last_workers : g.last_workers / g.warps_per_block;
        stats->block = g.cfg.block;
        stats->workers = g.last_workers;
        stats->status = st;
        stats->launches = launches;
        stats->light_workers = light_workers;
        stats->light_kernel_ms = ms_light;
    }
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// host-buffer entry point
// ---------------------------------------------------------------------------
namespace {
// One root array of a host-buffer batch and its place in the device slab.
struct HostCopy {
    void* host;   // null: device scratch only
    size_t off;
    size_t bytes;
    bool in;      // copied host -> device before the root runs
    bool out;     // copied device -> host after it ran
    bool sort;    // belongs to a sort root
};

// Slab layout: arrays of one class (sort or not, in / out / in-out /
// scratch) in plan order, and an array that continues the previous one of
// its class in host memory continues it in the slab too, so that a batch whose
// roots slice one host buffer moves it in one copy each way.  Other arrays
// start on 256-byte boundaries.  Returns the slab size.
size_t layout_slab(std::vector<HostCopy>& copies) {
    size_t total = 0;
    for (int cls = 0; cls < 8; ++cls) {
        const HostCopy* prev = nullptr;
        for (auto& c : copies) {
            const int k = (c.sort ? 4 : 0) + (c.in ? 2 : 0) + (c.out ? 1 : 0);
            if (k != cls) continue;
            const bool follows = prev && c.host && prev->host &&
                                 static_cast<const char*>(prev->host) + prev->bytes == c.host &&
                                 prev->off + prev->bytes == total;
            c.off = follows ? total : (total + 255) & ~(size_t)255;
            total = c.off + c.bytes;
            prev = &c;
        }
    }
    return total;
}

// Issue the copies of one direction and class, one per run of arrays that
// are contiguous on both sides.
int issue_copies(const std::vector<HostCopy>& copies, char* slab, bool to_device, bool sort, cudaStream_t s,
                 int64_t& bytes) {
    size_t run_off = 0, run_bytes = 0;
    const char* run_host = nullptr;
    auto flush = [&]() -> int {
        if (!run_bytes) return 0;
        cudaError_t e = to_device ? cudaMemcpyAsync(slab + run_off, run_host, run_bytes, cudaMemcpyHostToDevice, s)
                                  : cudaMemcpyAsync(const_cast<char*>(run_host), slab + run_off, run_bytes,
                                                    cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return -(int)e;
        bytes += (int64_t)run_bytes;
        run_bytes = 0;
        return 0;
    };
    for (int cls = 0; cls < 8; ++cls) {   // the layout's order, so that runs meet
        for (const auto& c : copies) {
            const int k = (c.sort ? 4 : 0) + (c.in ? 2 : 0) + (c.out ? 1 : 0);
            if (k != cls || c.sort != sort || !(to_device ? c.in : c.out)) continue;
            const char* h = static_cast<const char*>(c.host);
            if (run_bytes && run_host + run_bytes == h && run_off + run_bytes == c.off) {
                run_bytes += c.bytes;
                continue;
            }
            int rc = flush();
            if (rc) return rc;
            run_host = h;
            run_off = c.off;
            run_bytes = c.bytes;
        }
        int rc = flush();
        if (rc) return rc;
    }
    return 0;
}
}  // namespace

extern "C" int gtap_run_host(const gtap_root* roots, int32_t n_roots, gtap_root_result* results,
                             gtap_run_stats* stats, int64_t* h2d_bytes, int64_t* d2h_bytes) {
    if (!roots || n_roots < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.serving) return GTAP_ERROR_BUSY;
    std::vector<gtap_root> dev_roots(roots, roots + n_roots);
    std::vector<HostCopy> copies;
    bool sort_root = false;
    auto plan = [&](void* host, size_t bytes, bool in, bool out) -> int {
        copies.push_back(HostCopy{host, 0, bytes, in && host != nullptr, out && host != nullptr, sort_root});
        return (int)copies.size() - 1;
    };
    std::vector<std::vector<int>> idx(n_roots);
    for (int i = 0; i < n_roots; ++i) {
        const gtap_root& r = roots[i];
        sort_root = is_sort_kind(r.kind);
        switch (r.kind) {
            case GTAP_KIND_CILKSORT:
            case GTAP_KIND_MERGESORT: {
                size_t b = (size_t)r.n * sizeof(int);
                idx[i] = {plan(r.p0, b, true, false), plan(r.p1, b, false, true), plan(nullptr, b, false, false)};
                break;
            }
            case GTAP_KIND_BFS: {
                size_t nv = (size_t)r.n;
                const int* row = reinterpret_cast<const int*>(r.p0);
                size_t ne = (size_t)row[nv];
                idx[i] = {plan(r.p0, (nv + 1) * sizeof(int), true, false), plan(r.p1, ne * sizeof(int), true, false),
                          plan(r.p2, nv * sizeof(int), true, true)};
                break;
            }
            case GTAP_KIND_TREESUM: {
                size_t nn = (size_t)r.n * sizeof(int);
                idx[i] = {plan(r.p0, nn, true, false), plan(r.p1, nn, true, false), plan(r.p2, nn, true, false),
                          plan(r.p3, nn, true, false)};
                break;
            }
            default:
                break;
        }
    }
    const size_t total = layout_slab(copies);
    if (total > g_slab_bytes) {
        if (g_slab) cudaFree(g_slab);
        g_slab = nullptr;
        g_slab_bytes = 0;
        cudaError_t e = cudaMalloc(&g_slab, total);
        if (e != cudaSuccess) return -(int)e;
        g_slab_bytes = total;
    }
    for (int i = 0; i < n_roots; ++i) {
        gtap_root& r = dev_roots[i];
        const std::vector<int>& k = idx[i];
        void** ps[4] = {&r.p0, &r.p1, &r.p2, &r.p3};
        for (size_t j = 0; j < k.size(); ++j) *ps[j] = g_slab + copies[k[j]].off;
    }

    // the other roots' inputs on the launch stream; the sorts' inputs and
    // outputs on a copy stream that runs beside the launches (the copies
    // overlap them when the host buffers are pinned)
    int64_t hin = 0, hout = 0;
    cudaStream_t s = nullptr, cs = nullptr;
    cudaEvent_t in_done = nullptr, sorted = nullptr;
    GT_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    GT_CUDA(cudaEventCreateWithFlags(&in_done, cudaEventDisableTiming));
    GT_CUDA(cudaEventCreateWithFlags(&sorted, cudaEventDisableTiming));
    int st = 0;
    bool inputs_in = false;   // no output is copied back unless its inputs went in
    {
        BatchHooks hooks;
        hooks.before_launches = [&]() -> int {
            int rc = issue_copies(copies, g_slab, true, false, s, hin);
            if (rc == 0) rc = issue_copies(copies, g_slab, true, true, cs, hin);
            if (rc == 0 && cudaEventRecord(in_done, cs) != cudaSuccess) rc = GTAP_ERROR_INVALID_ARGUMENT;
            inputs_in = rc == 0;
            return rc;
        };
        hooks.sort_inputs = in_done;
        hooks.halve_light = true;
        hooks.after_sorts = [&]() -> int {
            if (cudaEventRecord(sorted, s) != cudaSuccess || cudaStreamWaitEvent(cs, sorted, 0) != cudaSuccess)
                return GTAP_ERROR_INVALID_ARGUMENT;
            return issue_copies(copies, g_slab, false, true, cs, hout);
        };
        st = run_batch(dev_roots.data(), n_roots, results, stats, s, &hooks);
        // sorts that never ran (a failed earlier launch) leave their outputs unwritten
    }
    if (inputs_in) {
        int oc = issue_copies(copies, g_slab, false, false, s, hout);
        if (st == 0) st = oc;
    }
    cudaError_t e = cudaStreamSynchronize(s);
    cudaError_t e2 = cudaStreamSynchronize(cs);
    cudaStreamDestroy(cs);
    cudaEventDestroy(in_done);
    cudaEventDestroy(sorted);
    hin += (int64_t)sizeof(gtap_root) * n_roots;
    if (results) hout += (int64_t)sizeof(gtap_root_result) * n_roots;
    if (h2d_bytes) *h2d_bytes = hin;
    if (d2h_bytes) *d2h_bytes = hout;
    if (e != cudaSuccess && st == 0) return -(int)e;
    if (e2 != cudaSuccess && st == 0) return -(int)e2;
    return st;
}

// ---------------------------------------------------------------------------
// serve mode
// ---------------------------------------------------------------------------
extern "C" int gtap_serve_start(int32_t ring_capacity, int32_t admit_watermark) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.serving) return GTAP_ERROR_BUSY;
    if (ring_capacity < 1 || admit_watermark < 0) return GTAP_ERROR_INVALID_ARGUMENT;
    int rc = ensure_root_capacity(ring_capacity);
    if (rc) return rc;
    g.serve_ring_cap = ring_capacity;
    g.done_cap = (unsigned)ring_capacity;
    GT_CUDA(cudaHostAlloc(&g.h_done_ring, sizeof(unsigned long long) * g.done_cap, cudaHostAllocMapped));
    memset(g.h_done_ring, 0, sizeof(unsigned long long) * g.done_cap);
    GT_CUDA(cudaHostGetDevicePointer(&g.d_done_ring, g.h_done_ring, 0));
    GT_CUDA(cudaHostAlloc(&g.h_pub_src, sizeof(unsigned) * 2, cudaHostAllocDefault));
    GT_CUDA(cudaHostAlloc(&g.h_shutdown_src, sizeof(int) * 2, cudaHostAllocDefault));
    GT_CUDA(cudaStreamCreateWithFlags(&g.serve_stream, cudaStreamNonBlocking));
    GT_CUDA(cudaStreamCreateWithFlags(&g.feed_stream, cudaStreamNonBlocking));
    GT_CUDA(cudaEventCreate(&g.serve_ev0));
    GT_CUDA(cudaEventCreate(&g.serve_ev1));
    if (g.h_report) memset(g.h_report, 0, sizeof(GtapErrorReport));
    // serve mode runs the light kernel (fib, n-queens, BFS and tree roots), or
    // the block kernel in block mode (every kind)
    const int W = block_mode() ? g.workers_block : g.workers_light;
    g.last_workers = W;
    g.last_block = block_mode();
    Arena A = make_arena(ring_capacity, 2, W);
    A.admit_watermark = admit_watermark > 0 ? admit_watermark : admission_watermark(W);
    reset_kernel<<<64, 256, 0, g.serve_stream>>>(A, g.counters, ring_capacity, W * g.cfg.ids_per_worker);
    GT_CUDA(cudaGetLastError());
    GT_CUDA(cudaEventRecord(g.serve_ev0, g.serve_stream));
    GT_CUDA(launch_worker(A, true, g.serve_stream));
    GT_CUDA(cudaEventRecord(g.serve_ev1, g.serve_stream));
    g.serve_published = 0;
    g.serve_polled = 0;
    g.serving = true;
    return 0;
}

extern "C" int gtap_serve_enqueue(const gtap_root* roots, int32_t n, int32_t* first_index) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.serving) return GTAP_ERROR_NOT_INITIALIZED;
    if (!roots || n < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    // a slot may be reused only after its previous root completed and was polled
    if ((long long)g.serve_published + n - g.serve_polled > g.serve_ring_cap) return GTAP_ERROR_QUEUE_OVERFLOW;
    unsigned first = g.serve_published;
    int done = 0;
    while (done < n) {
        unsigned slot = (first + done) % (unsigned)g.serve_ring_cap;
        int chunk = std::min<int>(n - done, g.serve_ring_cap - (int)slot);
        GT_CUDA(cudaMemcpyAsync(g.d_roots + slot, roots + done, sizeof(gtap_root) * chunk, cudaMemcpyHostToDevice,
                                g.feed_stream));
        done += chunk;
    }
    g.serve_published = first + (unsigned)n;
    g.h_pub_src[0] = g.serve_published;
    GT_CUDA(cudaMemcpyAsync(g.counters + kCtrPublished, g.h_pub_src, sizeof(unsigned), cudaMemcpyHostToDevice,
                            g.feed_stream));
    GT_CUDA(cudaStreamSynchronize(g.feed_stream));
    if (first_index) *first_index = (int32_t)first;
    return 0;
}

extern "C" int gtap_serve_poll(int32_t* indices, int32_t max, int32_t* n_out) {
    if (!g.serving) return GTAP_ERROR_NOT_INITIALIZED;
    if (!indices || !n_out || max < 0) return GTAP_ERROR_INVALID_ARGUMENT;
    int n = 0;
    while (n < max) {
        unsigned pos = g.serve_polled;
        volatile unsigned long long* p = g.h_done_ring + (pos % g.done_cap);
        unsigned long long w = *p;
        if ((unsigned)(w & 0xFFFFFFFFu) == 0 || (unsigned)(w >> 32) != pos) break;
        indices[n++] = (int32_t)((unsigned)(w & 0xFFFFFFFFu) - 1);
        g.serve_polled = pos + 1;
    }
    *n_out = n;
    // surface device errors without blocking
    if (g.h_report && g.h_report->valid) return g.h_report->code;
    return 0;
}

extern "C" int gtap_serve_results(const int32_t* indices, int32_t n, gtap_root_result* out) {
    if (!g.serving && !g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (!indices || !out || n < 0) return GTAP_ERROR_INVALID_ARGUMENT;
    // while serving, beside the running kernel; after shutdown, on the default stream
    cudaStream_t s = g.serving ? g.feed_stream : nullptr;
    for (int i = 0; i < n; ++i) {
        int slot = indices[i];
        if (slot < 0 || slot >= g.root_cap) return GTAP_ERROR_INVALID_ARGUMENT;
        GT_CUDA(cudaMemcpyAsync(out + i, g.d_results + slot, sizeof(gtap_root_result), cudaMemcpyDeviceToHost, s));
    }
    GT_CUDA(cudaStreamSynchronize(s));
    return 0;
}

extern "C" int gtap_serve_shutdown(gtap_run_stats* stats) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.serving) return GTAP_ERROR_NOT_INITIALIZED;
    g.h_shutdown_src[0] = 1;
    cudaMemcpyAsync(g.counters + kCtrShutdown, g.h_shutdown_src, sizeof(int), cudaMemcpyHostToDevice, g.feed_stream);
    cudaStreamSynchronize(g.feed_stream);
    cudaError_t e = cudaEventSynchronize(g.serve_ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g.serve_ev0, g.serve_ev1);
    g.serving = false;
    int st = (e == cudaSuccess) ? read_status() : -(int)e;
    if (stats) {
        collect_stats(stats);
        stats->kernel_ms = ms;
        stats->status = st;
    }
    cudaEventDestroy(g.serve_ev0);
    cudaEventDestroy(g.serve_ev1);
    cudaStreamDestroy(g.serve_stream);
    cudaStreamDestroy(g.feed_stream);
    g.serve_stream = nullptr;
    g.feed_stream = nullptr;
    g.serve_ev0 = nullptr;
    g.serve_ev1 = nullptr;
    cudaFreeHost(g.h_done_ring);
    cudaFreeHost(g.h_pub_src);
    cudaFreeHost(g.h_shutdown_src);
    g.h_done_ring = nullptr;
    g.d_done_ring = nullptr;
    g.h_pub_src = nullptr;
    g.h_shutdown_src = nullptr;
    return st;
}

// ---------------------------------------------------------------------------
// profiler CSVs (schema of runtime/detail/thread/gtap_profile_thread.cuh:29-108, 188-268)
// ---------------------------------------------------------------------------
namespace {
void ensure_dir(const char* path) {
    struct stat st {};
    if (stat(path, &st) == -1 && errno == ENOENT) mkdir(path, 0755);
}
}  // namespace

extern "C" int gtap_write_profile(const char* directory, const char* app_name) {
    if (!g.initialized || !g.have_profile || !directory || !app_name) return GTAP_ERROR_INVALID_ARGUMENT;
    // one row per worker of the last launch (warps, or blocks in block mode)
    const int W = g.last_workers > 0 ? std::min(g.last_workers, g.workers) : g.workers, P = g.cfg.profile_samples;
    std::vector<long long> hv((size_t)W * P), wv((size_t)W * P);
    std::vector<int> tv((size_t)W * P);
    GT_CUDA(cudaMemcpy(hv.data(), g.prof_having, hv.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    GT_CUDA(cudaMemcpy(wv.data(), g.prof_working, wv.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    GT_CUDA(cudaMemcpy(tv.data(), g.prof_tasks, tv.size() * sizeof(int), cudaMemcpyDeviceToHost));
    ensure_dir(directory);
    const char* unit = g.cfg.mode == GTAP_MODE_BLOCK ? "block" : "warp";
    long long tmin = LLONG_MAX;
    for (long long t : hv)
        if (t > 0 && t < tmin) tmin = t;
    for (long long t : wv)
        if (t > 0 && t < tmin) tmin = t;
    if (tmin == LLONG_MAX) tmin = 0;
    char path[1024];
    // having-task timeline + statistics
    snprintf(path, sizeof(path), "%s/%s_%s_timeline_having_task.csv", directory, app_name, unit);
    FILE* f = fopen(path, "w");
    if (!f) return GTAP_ERROR_INVALID_ARGUMENT;
    fprintf(f, "%s_id,time_index,timestamp_ns,relative_time_ms,state,state_description\n", unit);
    for (int w = 0; w < W; ++w) {
        std::vector<std::pair<long long, int>> e;
        for (int i = 0; i < P; ++i) {
            long long t = hv[(size_t)w * P + i];
            if (t > 0) e.push_back({t, i});
        }
        std::stable_sort(e.begin(), e.end());
        for (auto& x : e) {
            int state = (x.second % 2 == 0) ? 1 : 0;
            fprintf(f, "%d,%d,%lld,%.6f,%d,%s\n", w, x.second, x.first, (x.first - tmin) / 1e6, state,
                    state ? "Having" : "NotHaving");
        }
    }
    fclose(f);
    snprintf(path, sizeof(path), "%s/%s_%s_statistics_having_task.csv", directory, app_name, unit);
    f = fopen(path, "w");
    if (!f) return GTAP_ERROR_INVALID_ARGUMENT;
    fprintf(f, "%s_id,total_samples,first_activity_ms,last_activity_ms,duration_ms\n", unit);
    for (int w = 0; w < W; ++w) {
        int having = 0;
        long long first = LLONG_MAX, last = 0;
        for (int i = 0; i < P; ++i) {
            long long t = hv[(size_t)w * P + i];
            if (t > 0) {
                first = std::min(first, t);
                last = std::max(last, t);
                if (i % 2 == 0) ++having;
            }
        }
        if (last == 0) fprintf(f, "%d,0,0.0,0.0,0.0\n", w);
        else fprintf(f, "%d,%d,%.6f,%.6f,%.6f\n", w, having, (first - tmin) / 1e6, (last - tmin) / 1e6, (last - first) / 1e6);
    }
    fclose(f);
    // working timeline + statistics
    snprintf(path, sizeof(path), "%s/%s_%s_timeline_working.csv", directory, app_name, unit);
    f = fopen(path, "w");
    if (!f) return GTAP_ERROR_INVALID_ARGUMENT;
    fprintf(f, "%s_id,time_index,timestamp_ns,relative_time_ms,state,state_description,tasks_in_batch\n", unit);
    for (int w = 0; w < W; ++w) {
        for (int i = 0; i < P; ++i) {
            long long t = wv[(size_t)w * P + i];
            if (t <= 0) continue;
            int state = (i % 2 == 0) ? 1 : 0;
            fprintf(f, "%d,%d,%lld,%.6f,%d,%s,%d\n", w, i, t, (t - tmin) / 1e6, state, state ? "Working" : "NotWorking",
                    tv[(size_t)w * P + i]);
        }
    }
    fclose(f);
    snprintf(path, sizeof(path), "%s/%s_%s_statistics_working.csv", directory, app_name, unit);
    f = fopen(path, "w");
    if (!f) return GTAP_ERROR_INVALID_ARGUMENT;
    fprintf(f, "%s_id,total_samples,first_activity_ms,last_activity_ms,duration_ms,total_tasks\n", unit);
    for (int w = 0; w < W; ++w) {
        int working = 0;
        long long tasks = 0, first = LLONG_MAX, last = 0;
        for (int i = 0; i < P; ++i) {
            long long t = wv[(size_t)w * P + i];
            if (t > 0) {
                first = std::min(first, t);
                last = std::max(last, t);
                if (i % 2 == 0) {
                    ++working;
                    tasks += tv[(size_t)w * P + i];
                }
            }
        }
        if (last == 0) fprintf(f, "%d,0,0.0,0.0,0.0,0\n", w);
        else fprintf(f, "%d,%d,%.6f,%.6f,%.6f,%lld\n", w, working, (first - tmin) / 1e6, (last - tmin) / 1e6,
                     (last - first) / 1e6, tasks);
    }
    fclose(f);
    return 0;
}

extern "C" int gtap_visualize_profile(const char* app_name) { return gtap_write_profile("./profile", app_name); }

// ---------------------------------------------------------------------------
// generators
// ---------------------------------------------------------------------------
extern "C" int gtap_gen_keys(uint32_t seed, int32_t* out, int64_t n) {
    if (!out || n < 0) return GTAP_ERROR_INVALID_ARGUMENT;
    std::mt19937 rng(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = static_cast<int32_t>(rng());
    return 0;
}

extern "C" int gtap_gen_mix(uint64_t seed, int32_t n_roots, int32_t* kind, int32_t* param, uint64_t* key_seed) {
    if (n_roots < 0 || !kind || !param || !key_seed) return GTAP_ERROR_INVALID_ARGUMENT;
    std::mt19937_64 rng(seed);
    for (int32_t i = 0; i < n_roots; ++i) {
        uint64_t d0 = rng(), d1 = rng(), d2 = rng();
        int32_t k = (int32_t)(d0 % 3);
        kind[i] = k;
        if (k == 0) param[i] = 18 + (int32_t)(d1 % 11);
        else if (k == 1) param[i] = 8 + (int32_t)(d1 % 4);
        else param[i] = (int32_t)((1024 + (d1 >> 8) % 1024) << (d1 % 10));
        key_seed[i] = d2;
    }
    return 0;
}

extern "C" int gtap_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed, int32_t* row, int32_t* col) {
    if (scale < 1 || scale > 26 || edge_factor < 1 || !row || !col) return GTAP_ERROR_INVALID_ARGUMENT;
    const int64_t nv = (int64_t)1 << scale, ne = nv * edge_factor;
    std::vector<uint64_t> keys((size_t)ne);
    std::mt19937_64 rng(seed);
    for (int64_t e = 0; e < ne; ++e) {
        uint64_t src = 0, dst = 0;
        for (int lvl = 0; lvl < scale; ++lvl) {
            uint64_t r = rng() % 100;
            uint64_t sb = (r >= 76) ? 1 : 0;               // c (76..94) and d (95..99)
            uint64_t db = (r >= 57 && r < 76) || r >= 95;   // b (57..75) and d
            src = (src << 1) | sb;
            dst = (dst << 1) | db;
        }
        keys[(size_t)e] = (src << 32) | dst;
    }
    std::sort(keys.begin(), keys.end());
    std::fill(row, row + nv + 1, 0);
    for (int64_t e = 0; e < ne; ++e) {
        row[(keys[(size_t)e] >> 32) + 1]++;
        col[e] = (int32_t)(keys[(size_t)e] & 0xFFFFFFFFu);
    }
    for (int64_t v = 0; v < nv; ++v) row[v + 1] += row[v];
    return 0;
}

// ---------------------------------------------------------------------------
// on-disk formats of the reference's inputs
// ---------------------------------------------------------------------------
namespace {
struct File {
    FILE* f;
    explicit File(FILE* p) : f(p) {}
    ~File() {
        if (f) fclose(f);
    }
};
long long file_bytes(FILE* f) {
    if (fseek(f, 0, SEEK_END) != 0) return -1;
    const long long b = ftell(f);
    if (fseek(f, 0, SEEK_SET) != 0) return -1;
    return b;
}
}  // namespace

// evaluation/util/gen_vector.c:21-60: size_t n, then n int32 values.
extern "C" int gtap_read_array_file(const char* path, int32_t* out, int64_t capacity, int64_t* n_out) {
    if (!path || !n_out || capacity < 0) return GTAP_ERROR_INVALID_ARGUMENT;
    File fp(fopen(path, "rb"));
    if (!fp.f) return GTAP_ERROR_INVALID_ARGUMENT;
    const long long bytes = file_bytes(fp.f);
    uint64_t n = 0;
    if (bytes < 8 || fread(&n, sizeof(n), 1, fp.f) != 1) return GTAP_ERROR_INVALID_ARGUMENT;
    if (n > (uint64_t)INT64_MAX / 4 || (long long)(8 + 4 * n) != bytes) return GTAP_ERROR_INVALID_ARGUMENT;
    *n_out = (int64_t)n;
    if (!out) return 0;   // size query
    if ((uint64_t)capacity < n) return GTAP_ERROR_INVALID_ARGUMENT;
    if (n && fread(out, sizeof(int32_t), n, fp.f) != n) return GTAP_ERROR_INVALID_ARGUMENT;
    return 0;
}

extern "C" int gtap_write_array_file(const char* path, const int32_t* data, int64_t n) {
    if (!path || n < 0 || (n > 0 && !data)) return GTAP_ERROR_INVALID_ARGUMENT;
    File fp(fopen(path, "wb"));
    if (!fp.f) return GTAP_ERROR_INVALID_ARGUMENT;
    const uint64_t un = (uint64_t)n;
    if (fwrite(&un, sizeof(un), 1, fp.f) != 1) return GTAP_ERROR_INVALID_ARGUMENT;
    if (n && fwrite(data, sizeof(int32_t), (size_t)n, fp.f) != (size_t)n) return GTAP_ERROR_INVALID_ARGUMENT;
    return 0;
}

// examples/asynchronous_bfs/asynchronous_bfs_thread.cu:69-84: int N, int M,
// int row[N+1], int col[M].  The offsets must start at 0, never decrease and
// end at M, and every column must name a vertex.
extern "C" int gtap_read_csr_file(const char* path, int32_t* row, int64_t row_capacity, int32_t* col,
                                  int64_t col_capacity, int32_t* n_out, int32_t* m_out) {
    if (!path || !n_out || !m_out) return GTAP_ERROR_INVALID_ARGUMENT;
    File fp(fopen(path, "rb"));
    if (!fp.f) return GTAP_ERROR_INVALID_ARGUMENT;
    const long long bytes = file_bytes(fp.f);
    int32_t hdr[2];
    if (bytes < 8 || fread(hdr, sizeof(int32_t), 2, fp.f) != 2) return GTAP_ERROR_INVALID_ARGUMENT;
    const int32_t N = hdr[0], M = hdr[1];
    if (N < 0 || M < 0 || 8 + 4 * ((long long)N + 1 + M) != bytes) return GTAP_ERROR_INVALID_ARGUMENT;
    *n_out = N;
    *m_out = M;
    if (!row && !col) return 0;   // size query
    if (!row || !col || row_capacity < (int64_t)N + 1 || col_capacity < M) return GTAP_ERROR_INVALID_ARGUMENT;
    if (fread(row, sizeof(int32_t), (size_t)N + 1, fp.f) != (size_t)N + 1) return GTAP_ERROR_INVALID_ARGUMENT;
    if (M && fread(col, sizeof(int32_t), (size_t)M, fp.f) != (size_t)M) return GTAP_ERROR_INVALID_ARGUMENT;
    if (row[0] != 0 || row[N] != M) return GTAP_ERROR_INVALID_ARGUMENT;
    for (int32_t v = 0; v < N; ++v)
        if (row[v + 1] < row[v]) return GTAP_ERROR_INVALID_ARGUMENT;
    for (int32_t e = 0; e < M; ++e)
        if (col[e] < 0 || col[e] >= N) return GTAP_ERROR_INVALID_ARGUMENT;
    return 0;
}

extern "C" int gtap_write_csr_file(const char* path, const int32_t* row, const int32_t* col, int32_t n, int32_t m) {
    if (!path || n < 0 || m < 0 || !row || (m > 0 && !col)) return GTAP_ERROR_INVALID_ARGUMENT;
    File fp(fopen(path, "wb"));
    if (!fp.f) return GTAP_ERROR_INVALID_ARGUMENT;
    const int32_t hdr[2] = {n, m};
    if (fwrite(hdr, sizeof(int32_t), 2, fp.f) != 2) return GTAP_ERROR_INVALID_ARGUMENT;
    if (fwrite(row, sizeof(int32_t), (size_t)n + 1, fp.f) != (size_t)n + 1) return GTAP_ERROR_INVALID_ARGUMENT;
    if (m && fwrite(col, sizeof(int32_t), (size_t)m, fp.f) != (size_t)m) return GTAP_ERROR_INVALID_ARGUMENT;
    return 0;
}

extern "C" int gtap_gen_tree(int32_t n, uint64_t seed, int32_t* left, int32_t* right, int32_t* value, int32_t* size) {
    if (n < 1 || !left || !right || !value || !size) return GTAP_ERROR_INVALID_ARGUMENT;
    std::mt19937_64 rng(seed);
    std::vector<int32_t> pl(n), pr(n), pv(n), ps(n);
    std::vector<std::pair<int32_t, int32_t>> stack;   // (budget, preorder position)
    stack.push_back({n, 0});
    while (!stack.empty()) {
        auto [b, i] = stack.back();
        stack.pop_back();
        pv[i] = (int32_t)(uint32_t)rng();
        int32_t L = 0;
        for (int32_t k = 0; k < b - 1; ++k)
            if (rng() % 100 < 48) ++L;
        int32_t R = b - 1 - L;
        ps[i] = b;
        pl[i] = L > 0 ? i + 1 : -1;
        pr[i] = R > 0 ? i + 1 + L : -1;
        if (R > 0) stack.push_back({R, i + 1 + L});
        if (L > 0) stack.push_back({L, i + 1});
    }
    std::vector<int32_t> perm(n);
    for (int32_t i = 0; i < n; ++i) perm[i] = i;
    for (int32_t i = n - 1; i >= 2; --i) {
        int32_t j = 1 + (int32_t)(rng() % (uint64_t)i);
        std::swap(perm[i], perm[j]);
    }
    for (int32_t i = 0; i < n; ++i) {
        int32_t p = perm[i];
        left[p] = pl[i] >= 0 ? perm[pl[i]] : -1;
        right[p] = pr[i] >= 0 ? perm[pr[i]] : -1;
        value[p] = pv[i];
        size[p] = ps[i];
    }
    return 0;
}

// ---------------------------------------------------------------------------
// queue self-test
// ---------------------------------------------------------------------------
namespace {
__global__ void selftest_count_kernel(const unsigned* seen, size_t n, unsigned long long* ones,
                                      unsigned long long* dups) {
    unsigned long long o = 0, d = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned v = seen[i];
        o += (v == 1u);
        d += (v > 1u) ? (v - 1u) : 0u;
    }
    atomicAdd(ones, o);
    atomicAdd(dups, d);
}
}  // namespace

extern "C" int gtap_selftest_queues(int32_t rounds, int32_t per_round_max, int32_t mode, int64_t* produced,
                                    int64_t* consumed, int64_t* duplicates, int64_t* lost) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.serving) return GTAP_ERROR_BUSY;
    if (rounds < 1 || per_round_max < 0 || per_round_max > g.cfg.spawn_capacity || mode < 0 || mode > 7)
        return GTAP_ERROR_INVALID_ARGUMENT;
    const int W = g.workers_light;
    const size_t ntok = (size_t)W * 16384;
    // every token may sit in the overflow ring at once: keep the volume below its capacity
    if ((long long)rounds * per_round_max > 16383 ||
        (long long)W * rounds * per_round_max > (1ll << g.overflow_log2))
        return GTAP_ERROR_INVALID_ARGUMENT;
    unsigned* seen = nullptr;
    SelftestCounters* ctr = nullptr;
    unsigned long long* sums = nullptr;
    GT_CUDA(cudaMalloc(&seen, ntok * sizeof(unsigned)));
    GT_CUDA(cudaMemset(seen, 0, ntok * sizeof(unsigned)));
    GT_CUDA(cudaMalloc(&ctr, sizeof(SelftestCounters)));
    GT_CUDA(cudaMemset(ctr, 0, sizeof(SelftestCounters)));
    GT_CUDA(cudaMalloc(&sums, 2 * sizeof(unsigned long long)));
    GT_CUDA(cudaMemset(sums, 0, 2 * sizeof(unsigned long long)));
    Arena A = make_arena(1, 0, W);
    reset_kernel<<<64, 256>>>(A, g.counters, 1, W * g.cfg.ids_per_worker);
    GT_CUDA(cudaGetLastError());
    GT_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(&selftest_queue_kernel),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem_bytes));
    selftest_queue_kernel<<<W / g.warps_per_block, g.cfg.block, g.smem_bytes>>>(A, rounds, per_round_max, seen, ctr,
                                                                                 mode);
    GT_CUDA(cudaGetLastError());
    selftest_count_kernel<<<1184, 256>>>(seen, ntok, sums, sums + 1);
    GT_CUDA(cudaDeviceSynchronize());
    SelftestCounters hc{};
    unsigned long long hs[2] = {0, 0};
    GT_CUDA(cudaMemcpy(&hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost));
    GT_CUDA(cudaMemcpy(hs, sums, sizeof(hs), cudaMemcpyDeviceToHost));
    cudaFree(seen);
    cudaFree(ctr);
    cudaFree(sums);
    const long long ones = (long long)hs[0], dups = (long long)hs[1];
    if (produced) *produced = hc.produced;
    if (consumed) *consumed = hc.consumed;
    if (duplicates) *duplicates = dups + hc.bad_tokens;
    if (lost) *lost = (long long)hc.produced - ones;
    int st = read_status();
    if (st) return st;
    return (dups == 0 && hc.bad_tokens == 0 && ones == (long long)hc.produced) ? 0 : GTAP_ERROR_QUEUE_OVERFLOW;
}

// ---------------------------------------------------------------------------
// testing aid: ring positions
// ---------------------------------------------------------------------------
namespace gtap {
int noalloc_set_ring_position(uint32_t position);   // gtap_noalloc.cu
}

extern "C" int gtap_debug_admission_order(const gtap_root* roots, int32_t n, int32_t* order, int32_t* n_light) {
    if (!roots || n < 0 || !order || !n_light) return GTAP_ERROR_INVALID_ARGUMENT;
    std::vector<int> o;
    *n_light = admission_order(roots, n, o);
    for (int i = 0; i < n; ++i) order[i] = o.empty() ? i : o[i];
    return 0;
}

extern "C" int gtap_debug_set_ring_position(int32_t target, uint32_t position) {
    if (target == 1) {
        std::lock_guard<std::mutex> lk(g_mu);
        return gtap::noalloc_set_ring_position(position);
    }
    if (target != 0) return GTAP_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    if (g.serving) return GTAP_ERROR_BUSY;
    GT_CUDA(cudaDeviceSynchronize());
    const unsigned pos[4] = {position, position, position, position};
    // kCtrOvHead, kCtrOvTail, kCtrPoolHead, kCtrPoolTail are adjacent
    static_assert(kCtrOvTail == kCtrOvHead + 1 && kCtrPoolHead == kCtrOvHead + 2 && kCtrPoolTail == kCtrOvHead + 3,
                  "ring cursor slots");
    GT_CUDA(cudaMemcpy(g.counters + kCtrOvHead, pos, sizeof(pos), cudaMemcpyHostToDevice));
    // the slots are cleared too: a slot's tag is its position's lap, so a
    // word left from before the jump could carry the tag of a position 2^32
    // further on (continuous use rewrites every slot once per lap instead)
    const size_t nslots = (1ull << g.overflow_log2) + (1ull << g.idpool_log2);
    GT_CUDA(cudaMemset(g.ring_slots, 0, nslots * sizeof(unsigned long long)));
    GT_CUDA(cudaDeviceSynchronize());
    return 0;
}

// ---------------------------------------------------------------------------
// arena counters after the last launch (task-id accounting)
// ---------------------------------------------------------------------------
extern "C" int gtap_get_arena_counters(int64_t* out, int32_t n) {
    if (!out || n < 8) return GTAP_ERROR_INVALID_ARGUMENT;
    if (!g.initialized) return GTAP_ERROR_NOT_INITIALIZED;
    unsigned h[kCtrCount];
    GT_CUDA(cudaMemcpy(h, g.counters, sizeof(h), cudaMemcpyDeviceToHost));
    out[0] = h[kCtrFresh];                                  // next never-used id
    out[1] = (long long)g.last_workers * g.cfg.ids_per_worker;   // first id outside the private ranges
    out[2] = (int64_t)(h[kCtrPoolTail] - h[kCtrPoolHead]);  // recycled ids waiting in the pool
    out[3] = (int64_t)(h[kCtrOvTail] - h[kCtrOvHead]);      // tasks left in the overflow queue
    out[4] = h[kCtrCompleted];
    out[5] = g.cfg.total_ids;
    out[6] = g.last_workers;
    out[7] = h[kCtrStatus];
    return 0;
}
