// gtap_noalloc.cu -- gtap_launch_noalloc: run roots without allocating memory.
//
// Some callers cannot call cudaMalloc: a serving loop that must not take the
// implicit device-wide synchronisation an allocation can cause, a process
// whose device memory already belongs to another allocator (a framework pool
// that reserved nearly all of HBM, where a fresh cudaMalloc fails or
// fragments), or a library embedded in such a host that is not allowed to
// change the device's memory footprint after start-up.  For them this entry
// point keeps all of the scheduler's working memory -- task records, deques,
// the overflow and recycled-id queues, counters and statistics -- in one
// file-scope device array of fixed size, kNoallocBytes (about 45 MiB).  Every
// GPU that loads the library holds that array until the process exits.
//
// The caller still owns the inputs and outputs: the root descriptors and the
// result array are device buffers it allocated, as are any arrays the roots
// point to (BFS graphs, trees).
//
// Limits:
//   * at most kNoallocMaxRoots (4096) roots per call, else GTAP_ERROR_INVALID_ARGUMENT;
//   * only the register-light kinds: fib, n-queens, BFS, tree sum (a sorting
//     root is refused on the device with GTAP_ERROR_INVALID_KIND);
//   * kNoallocIds (2^19) task records, shared by the tasks alive at once and
//     the free ids each worker keeps at hand; a tree that needs more is
//     reported as GTAP_ERROR_TASK_ID_POOL_LOW_HEADROOM by the device, not a
//     fault.  How many tasks are alive at once depends on the tree and the
//     schedule: a tree whose tasks create many children at once, such as
//     n-queens(16) with every row forking, exceeds it; a binary tree that
//     waits for its children keeps few alive (fib(34) without a cutoff
//     fits).
//
// Set-up: the first call on a device, with that device current, sizes the
// grid with an occupancy query.  Make that first call before any stream
// capture.  Every call, with its device current, then looks up the array's
// device address with cudaGetSymbolAddress (host code must not use the
// symbol itself: on the host it only names a stand-in, and a kernel given it
// would fault or read the wrong memory) and sets the kernel's shared-memory
// limit.  Both are cheap and allocate nothing; redoing them each call keeps a
// call correct after a cudaDeviceReset (a new context loads the module again,
// possibly at another address) and after gtap_initialize() set a different
// limit on the same kernel.
//
// The call is synchronous: it returns once the launch has finished, with the
// device status.  Calls from one process are serialised by a lock.  Every
// call uses the same array and it keeps the previous call's contents; each
// call clears what must start at zero.  Work that overlaps on the GPU and
// bypasses that lock (two processes sharing a context, or device code of
// another library writing the array) races on the array and corrupts it.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/gtap.h"
#include "gtap_programs.cuh"

using namespace gtap;

namespace gtap {
int noalloc_set_ring_position(uint32_t position);   // testing aid, called by gtap_debug_set_ring_position
}

namespace {

constexpr int kNoallocMaxWorkers = 1184;             // 148 SMs x 2 blocks x 4 warps
constexpr int kNoallocBlock = 128;                 // 4 warps per block
constexpr int kNoallocDequeLog2 = 10;              // 1024 slots per worker
constexpr int kNoallocIds = 1 << 19;               // task records
constexpr int kNoallocRingLog2 = 20;               // >= kNoallocIds + 1 slots per ring
constexpr int kNoallocMaxRoots = 4096;
constexpr int kNoallocIdsPerWorker = 128;
constexpr int kNoallocCacheIds = 64;               // free ids a worker keeps cached
constexpr int kNoallocSpawnCap = 512;
constexpr int kNoallocRecStride = kHdrBytes + 32;  // built-in frames are 32 bytes
constexpr int kNoallocCounters = 32;

constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }
constexpr size_t kOffRecords = 0;
constexpr size_t kOffCtl = align256(kOffRecords + (size_t)(kNoallocIds + 1) * kNoallocRecStride);
constexpr size_t kOffSlots = align256(kOffCtl + (size_t)kNoallocMaxWorkers * 8);
constexpr size_t kOffRings = align256(kOffSlots + ((size_t)kNoallocMaxWorkers << kNoallocDequeLog2) * 4);
constexpr size_t kOffCounters = align256(kOffRings + ((size_t)2 << kNoallocRingLog2) * 8);
constexpr size_t kOffHungry = align256(kOffCounters + (size_t)kNoallocCounters * 4);
constexpr size_t kOffStats = align256(kOffHungry + (size_t)kHungryReplicas * kHungryStride * 4);
constexpr size_t kOffOutstanding = align256(kOffStats + (size_t)kNoallocMaxWorkers * GTAP_STAT_COUNT * 8);
constexpr size_t kNoallocBytes = align256(kOffOutstanding + (size_t)kNoallocMaxRoots * 8);
static_assert((1u << kNoallocRingLog2) > (unsigned)kNoallocIds, "rings must hold every task id");

// counter slots inside the scratch array
enum { cFresh = 0, cOvHead, cOvTail, cPoolHead, cPoolTail, cNextRoot, cCompleted, cStatus, cAbort, cDone,
       cPublished, cShutdown, cLive, cHandleTop };

// The scratch.  Device code in this file could name it directly; host code
// only ever passes the address obtained from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

struct DeviceSetup {
    bool ready = false;
    int workers = 0;
    size_t smem = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_noalloc_mu;

size_t noalloc_smem() {
    const int wpb = kNoallocBlock / 32;
    return sizeof(WarpShared) * (size_t)wpb + (size_t)wpb * (kNoallocSpawnCap + kLocalCap) * sizeof(int);
}

__global__ void noalloc_reset_kernel(Arena A, unsigned* counters, int n_roots, int fresh_base) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int i = tid; i < A.num_workers; i += stride) A.dq_ctl[i] = 0ull;
    for (int i = tid; i < A.num_workers * GTAP_STAT_COUNT; i += stride) A.stats[i] = 0ull;
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
    // the ring cursors keep counting across calls (gtap_ring.h): queued
    // entries are dropped by moving each head to its tail
    for (int i = tid; i < kNoallocCounters; i += stride) {
        if (i == cOvTail || i == cPoolTail) continue;
        counters[i] = (i == cFresh) ? (unsigned)fresh_base
                      : (i == cOvHead) ? counters[cOvTail]
                      : (i == cPoolHead) ? counters[cPoolTail] : 0u;
    }
}

const void* noalloc_kernel() {
    return reinterpret_cast<const void*>(&thread_worker_kernel_lb<BuiltinProgramLight, 1>);
}

// Per call, with the device current: the array's device address in this
// context, and the kernel's shared-memory limit (gtap_initialize sets the same
// kernel's limit from its own configuration, which may be lower).
int bind_scratch(unsigned char** base) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return -(int)e;
    e = cudaFuncSetAttribute(noalloc_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)noalloc_smem());
    if (e != cudaSuccess) return -(int)e;
    *base = static_cast<unsigned char*>(ptr);
    return 0;
}

// Once per device: the grid (needs the shared-memory limit bound first).
int setup_device(int dev, DeviceSetup& d) {
    if (d.ready) return 0;
    const void* kfn = noalloc_kernel();
    const size_t smem = noalloc_smem();
    cudaError_t e;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kNoallocBlock, smem);
    if (e != cudaSuccess) return -(int)e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return -(int)e;
    if (per_sm < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    const int wpb = kNoallocBlock / 32;
    const int blocks = std::min(std::min(per_sm, 2) * sms, kNoallocMaxWorkers / wpb);
    d.workers = blocks * wpb;
    d.smem = smem;
    d.ready = true;
    return 0;
}

}  // namespace

// Testing aid behind gtap_debug_set_ring_position(1, pos): both rings empty
// with their cursors at `position` (the caller holds the library lock).
int gtap::noalloc_set_ring_position(uint32_t position) {
    unsigned char* base = nullptr;
    int rc = bind_scratch(&base);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    const unsigned pos[4] = {position, position, position, position};
    static_assert(cOvTail == cOvHead + 1 && cPoolHead == cOvHead + 2 && cPoolTail == cOvHead + 3, "ring cursors");
    cudaError_t e = cudaMemcpy(base + kOffCounters + sizeof(unsigned) * cOvHead, pos, sizeof(pos),
                               cudaMemcpyHostToDevice);
    // both rings' slots are cleared too (a word from before the jump could
    // carry the lap tag of a position 2^32 further on)
    if (e == cudaSuccess) e = cudaMemset(base + kOffRings, 0, ((size_t)2 << kNoallocRingLog2) * 8);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : -(int)e;
}

// See include/gtap.h.  No allocation: cudaGetSymbolAddress, attribute and
// occupancy queries, two kernel launches, one 4-byte status read.
extern "C" int gtap_launch_noalloc(const gtap_root* d_roots, int32_t n_roots, gtap_root_result* d_results,
                                   void* stream) {
    if (!d_roots || !d_results || n_roots < 1) return GTAP_ERROR_INVALID_ARGUMENT;
    if (n_roots > kNoallocMaxRoots) return GTAP_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return -(int)e;
    if (dev < 0 || dev >= kMaxDevices) return GTAP_ERROR_INVALID_ARGUMENT;
    DeviceSetup& d = g_setup[dev];
    unsigned char* base = nullptr;
    int rc = bind_scratch(&base);
    if (rc) return rc;
    rc = setup_device(dev, d);
    if (rc) return rc;

    unsigned* counters = reinterpret_cast<unsigned*>(base + kOffCounters);
    const int W = d.workers;

    Arena A{};
    A.num_workers = W;
    A.warps_per_block = kNoallocBlock / 32;
    A.num_queues = 1;
    A.deque_cap_log2 = kNoallocDequeLog2;
    A.steal_batch = 32;
    A.victim_policy = GTAP_VICTIM_PROBE_MAX;
    A.probe_width = 16;
    A.spawn_cap = kNoallocSpawnCap;
    A.ids_per_worker = kNoallocIdsPerWorker;
    A.avail_target = kNoallocCacheIds;
    A.rec_stride = kNoallocRecStride;
    A.admit_batch = 1;
    A.mode = 0;
    A.publish_lazy = 0;
    A.max_inflight = 0;
    A.total_ids = kNoallocIds;
    A.watchdog_ns = 20000ull * 1000000ull;
    A.records = reinterpret_cast<char*>(base + kOffRecords);
    A.funcs = nullptr;
    A.dq_ctl = reinterpret_cast<unsigned long long*>(base + kOffCtl);
    A.dq_slots = reinterpret_cast<int*>(base + kOffSlots);
    unsigned long long* rings = reinterpret_cast<unsigned long long*>(base + kOffRings);
    A.overflow.slots = rings;
    A.overflow.head = counters + cOvHead;
    A.overflow.tail = counters + cOvTail;
    A.overflow.cap_log2 = kNoallocRingLog2;
    A.idpool.slots = rings + (1ull << kNoallocRingLog2);
    A.idpool.head = counters + cPoolHead;
    A.idpool.tail = counters + cPoolTail;
    A.idpool.cap_log2 = kNoallocRingLog2;
    A.fresh_next = counters + cFresh;
    A.roots = d_roots;
    A.results = d_results;
    A.outstanding = reinterpret_cast<long long*>(base + kOffOutstanding);
    A.n_roots = n_roots;
    A.next_root = counters + cNextRoot;
    A.published = counters + cPublished;
    A.shutdown = reinterpret_cast<const int*>(counters + cShutdown);
    A.completed = counters + cCompleted;
    A.done_ring = nullptr;
    A.done_ring_cap = 0;
    A.live_tasks = reinterpret_cast<int*>(counters + cLive);
    A.admit_watermark = (kNoallocIds - W * kNoallocIdsPerWorker) / 4;
    A.status = reinterpret_cast<int*>(counters + cStatus);
    A.abort_flag = reinterpret_cast<int*>(counters + cAbort);
    A.done_flag = reinterpret_cast<int*>(counters + cDone);
    A.report = nullptr;
    A.dbg_live = nullptr;
    A.dbg_exec = nullptr;
    A.dbg_slotpos = nullptr;
    A.hungry = reinterpret_cast<int*>(base + kOffHungry);
    A.stats = reinterpret_cast<unsigned long long*>(base + kOffStats);
    A.prof_having = nullptr;
    A.prof_working = nullptr;
    A.prof_tasks = nullptr;
    A.prof_cap = 0;
    A.handles = nullptr;
    A.handle_top = reinterpret_cast<int*>(counters + cHandleTop);
    A.handle_meta = nullptr;
    A.handle_cap = 0;

    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    noalloc_reset_kernel<<<64, 256, 0, s>>>(A, counters, n_roots, W * kNoallocIdsPerWorker);
    e = cudaGetLastError();
    if (e != cudaSuccess) return -(int)e;
    thread_worker_kernel_lb<BuiltinProgramLight, 1><<<W / A.warps_per_block, kNoallocBlock, d.smem, s>>>(A);
    e = cudaGetLastError();
    if (e != cudaSuccess) return -(int)e;
    int status = 0;
    e = cudaMemcpyAsync(&status, counters + cStatus, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return -(int)e;
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return -(int)e;
    return status;
}
