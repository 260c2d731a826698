// gtap_microbench.cu -- the measured peak rate of the L2 atomics the
// scheduler issues, the denominator of its atomic roofline.
//
// The scheduler's atomics are 32-bit adds with a return value on scattered
// words that are rarely contended (a finishing task's decrement of its
// parent's join counter, one per task that has a waiting parent) plus CASes
// on per-worker deque words.  The kernel below issues the first kind at the
// highest rate the GPU allows: every thread of a full grid issues adds to
// pseudo-random words of a 64 MiB table (L2-resident on a B200), eight in
// flight per thread, and folds the returned values into one store so none
// can be elided.  mode 1 issues the same adds without a return value
// (red.add, what the root counters use).  Timed with CUDA events after a
// warm-up launch.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gtap.h"

namespace {

constexpr int kTableLog2 = 24;      // 2^24 words = 64 MiB
constexpr int kInFlight = 8;

__device__ __forceinline__ unsigned mix32(unsigned x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

template <int MODE>
__global__ void atomic_rate_kernel(int* table, int iters, unsigned long long* sink) {
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned mask = (1u << kTableLog2) - 1u;
    unsigned acc = 0;
    unsigned h = mix32(tid * 0x9E3779B9u + 1u);
    for (int it = 0; it < iters; ++it) {
        int* p[kInFlight];
#pragma unroll
        for (int j = 0; j < kInFlight; ++j) {
            h = mix32(h + (unsigned)j);
            p[j] = table + (h & mask);
        }
        if (MODE == 0) {
            int v[kInFlight];
#pragma unroll
            for (int j = 0; j < kInFlight; ++j)
                asm volatile("atom.relaxed.gpu.global.add.s32 %0, [%1], 1;" : "=r"(v[j]) : "l"(p[j]) : "memory");
#pragma unroll
            for (int j = 0; j < kInFlight; ++j) acc += (unsigned)v[j];
        } else {
#pragma unroll
            for (int j = 0; j < kInFlight; ++j)
                asm volatile("red.relaxed.gpu.global.add.s32 [%0], 1;" ::"l"(p[j]) : "memory");
        }
    }
    if (acc == 0xFFFFFFFFu) sink[0] = acc;   // keeps the returned values live
}

}  // namespace

extern "C" int gtap_measure_atomic_rate(int32_t mode, int64_t ops, double* ops_per_s) {
    if ((mode != 0 && mode != 1) || ops < (1 << 20) || !ops_per_s) return GTAP_ERROR_INVALID_ARGUMENT;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return -(int)e;
    int* table = nullptr;
    unsigned long long* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const int block = 256, grid = sms * 8;
    const long long per_launch_threads = (long long)grid * block;
    int iters = (int)((ops + per_launch_threads * kInFlight - 1) / (per_launch_threads * kInFlight));
    if (iters < 1) iters = 1;
    float ms = 0.f;
    if ((e = cudaMalloc(&table, sizeof(int) << kTableLog2)) != cudaSuccess) goto done;
    if ((e = cudaMalloc(&sink, sizeof(unsigned long long))) != cudaSuccess) goto done;
    if ((e = cudaMemset(table, 0, sizeof(int) << kTableLog2)) != cudaSuccess) goto done;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) goto done;
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) goto done;
    for (int rep = 0; rep < 2; ++rep) {   // the first launch warms L2 and the clocks
        cudaEventRecord(e0);
        if (mode == 0) atomic_rate_kernel<0><<<grid, block>>>(table, iters, sink);
        else atomic_rate_kernel<1><<<grid, block>>>(table, iters, sink);
        cudaEventRecord(e1);
        if ((e = cudaGetLastError()) != cudaSuccess) goto done;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) goto done;
    }
    cudaEventElapsedTime(&ms, e0, e1);
    *ops_per_s = (double)per_launch_threads * iters * kInFlight / (ms / 1e3);
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (table) cudaFree(table);
    if (sink) cudaFree(sink);
    return e == cudaSuccess ? 0 : -(int)e;
}
