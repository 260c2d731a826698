// cuda_runtime.h -- TEST INFRASTRUCTURE: a host stand-in for the few CUDA
// runtime calls, qualifiers and intrinsics that the pragma programs in
// tests/pragma use, so that their lowered text compiles with g++ and runs
// on the CPU under the task-ABI emulator in gtap_thread.cuh (this folder).
// Device memory is host memory; a kernel launch runs the kernel body as one
// block (the test rewrites `k<<<g, b>>>(args)` to `emu_launch([&] { k(args); })`):
// one thread in thread mode, a pool of threads in block mode, whose
// __syncthreads is a barrier; atomics are host atomics.
#pragma once
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __shared__ static
#define __constant__
#define __forceinline__ inline
#define __noinline__
#define __restrict__ __restrict
#define __launch_bounds__(...)

struct emu_dim3 {
    unsigned x, y, z;
};
static thread_local emu_dim3 threadIdx = {0, 0, 0};
static emu_dim3 blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1};

// threads that run each emulated block (1 in thread mode; the block-mode
// emulator sets it), and the barrier __syncthreads calls (none with one thread)
inline int& emu_block_threads() {
    static int t = 1;
    return t;
}
inline void (*&emu_sync_hook())() {
    static void (*h)() = nullptr;
    return h;
}
// a kernel launch: the kernel body on emu_block_threads() threads of one block
template <class F>
inline void emu_launch(F f) {
    const int T = emu_block_threads();
    blockDim.x = (unsigned)T;
    if (T == 1) {
        threadIdx.x = 0;
        f();
        return;
    }
    std::vector<std::thread> ts;
    for (int i = 0; i < T; ++i)
        ts.emplace_back([&f, i] {
            threadIdx.x = (unsigned)i;
            f();
        });
    for (auto& t : ts) t.join();
}

struct int4 {
    int x, y, z, w;
};
inline int4 make_int4(int x, int y, int z, int w) { return int4{x, y, z, w}; }

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice };
typedef int cudaEvent_t;

inline cudaError_t cudaMalloc(void** p, size_t n) {
    *p = malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
template <class T>
inline cudaError_t cudaMalloc(T** p, size_t n) { return cudaMalloc(reinterpret_cast<void**>(p), n); }
inline cudaError_t cudaFree(void* p) { free(p); return cudaSuccess; }
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) { memcpy(d, s, n); return cudaSuccess; }
inline cudaError_t cudaMemset(void* p, int v, size_t n) { memset(p, v, n); return cudaSuccess; }
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T& sym, const void* src, size_t n, size_t off = 0,
                                      cudaMemcpyKind = cudaMemcpyHostToDevice) {
    memcpy(reinterpret_cast<char*>(&sym) + off, src, n);
    return cudaSuccess;
}
template <class T>
inline cudaError_t cudaMemcpyFromSymbol(void* dst, const T& sym, size_t n, size_t off = 0,
                                        cudaMemcpyKind = cudaMemcpyDeviceToHost) {
    memcpy(dst, reinterpret_cast<const char*>(&sym) + off, n);
    return cudaSuccess;
}
inline cudaError_t cudaEventCreate(cudaEvent_t* e) { *e = 0; return cudaSuccess; }
inline cudaError_t cudaEventRecord(cudaEvent_t, int = 0) { return cudaSuccess; }
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t, cudaEvent_t) { *ms = 0.f; return cudaSuccess; }
inline cudaError_t cudaEventDestroy(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline const char* cudaGetErrorString(cudaError_t) { return "emulated"; }

inline int atomicAdd(int* p, int v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline unsigned atomicAdd(unsigned* p, unsigned v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
    return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
inline int atomicMin(int* p, int v) {
    int o = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (v < o && !__atomic_compare_exchange_n(p, &o, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
    }
    return o;
}
inline int atomicCAS(int* p, int expected, int desired) {
    __atomic_compare_exchange_n(p, &expected, desired, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return expected;
}
inline long long __double_as_longlong(double d) { long long r; memcpy(&r, &d, sizeof(r)); return r; }
inline int __ffsll(long long x) { return __builtin_ffsll(x); }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline void __threadfence() {}
inline void __syncthreads() {
    if (emu_sync_hook()) emu_sync_hook()();
}
