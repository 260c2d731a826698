// gtap_device_util.cuh -- the device helpers the reference's runtime headers
// expose to task code, under the same names and signatures.
//
// Programs written for the reference read shared data with these helpers
// (its cilksort and BFS examples call load_L2 on keys and on the visited
// array), so the drop-in headers gtap_thread.cuh and gtap_block.cuh include
// this file.  Reference: runtime/detail/common/gtap_runtime_common.cuh:89-204
// (L2 loads and stores, the acquire/release forms, lane and warp ids) and
// :246 (global time).
//
//   load_L2 / store_L2           a load or store that bypasses L1 (the .cg cache
//                                operator), so a value another SM wrote is seen
//   load_L2_acquire / store_L2_release   the same with gpu-scope acquire / release
//   load_L2_ptr / store_L2_ptr   pointer-sized forms
//   atomicCAS_acquire            compare-and-swap with gpu-scope acquire order
//   get_lane_id, get_warp_id_in_block, get_warp_id_global   for 1-D blocks
//   get_global_time              the %globaltimer nanosecond clock
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

__device__ __forceinline__ int load_L2(int* ptr) { return __ldcg(ptr); }
__device__ __forceinline__ unsigned int load_L2(unsigned int* ptr) { return __ldcg(ptr); }
__device__ __forceinline__ uint16_t load_L2_u16t(uint16_t* ptr) { return __ldcg(ptr); }

__device__ __forceinline__ int load_L2_acquire(int* ptr) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(ptr) : "memory");
    return v;
}

__device__ __forceinline__ void* load_L2_ptr(void** ptr) {
    return reinterpret_cast<void*>(__ldcg(reinterpret_cast<unsigned long long*>(ptr)));
}
template <typename T>
__device__ __forceinline__ T* load_L2_ptr(T** ptr) {
    return reinterpret_cast<T*>(load_L2_ptr(reinterpret_cast<void**>(ptr)));
}

__device__ __forceinline__ void store_L2(int* ptr, int val) { __stcg(ptr, val); }
__device__ __forceinline__ void store_L2(unsigned int* ptr, unsigned int val) { __stcg(ptr, val); }
__device__ __forceinline__ void store_L2_u16t(uint16_t* ptr, uint16_t val) { __stcg(ptr, val); }

__device__ __forceinline__ void store_L2_release(int* ptr, int val) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(ptr), "r"(val) : "memory");
}

__device__ __forceinline__ void store_L2_ptr(void** ptr, void* val) {
    __stcg(reinterpret_cast<unsigned long long*>(ptr), reinterpret_cast<unsigned long long>(val));
}
template <typename T>
__device__ __forceinline__ void store_L2_ptr(T** ptr, T* val) {
    store_L2_ptr(reinterpret_cast<void**>(ptr), reinterpret_cast<void*>(val));
}

__device__ __forceinline__ int atomicCAS_acquire(int* addr, int expected, int desired) {
    int old;
    asm volatile("atom.acquire.gpu.global.cas.b32 %0, [%1], %2, %3;"
                 : "=r"(old) : "l"(addr), "r"(expected), "r"(desired) : "memory");
    return old;
}

__device__ __forceinline__ unsigned int get_lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned int get_warp_id_in_block() { return threadIdx.x >> 5; }
__device__ __forceinline__ unsigned int get_warp_id_global() {
    return (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}

__device__ __forceinline__ unsigned long long get_global_time() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
