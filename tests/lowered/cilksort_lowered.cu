// cilksort_lowered.cu -- examples/cilksort/cilksort.cu:17-169 hand-lowered
// to the reference's task ABI: cilksort splits into four sorts, two merges
// and a final merge with three taskwaits; cilkmerge splits by a binary
// search until fewer than TASK_SPAWN_CUTOFF_MERGE keys remain; leaves below
// TASK_SPAWN_CUTOFF_SORT keys run a 64-key bitonic network in registers.
// Compiles against the reference runtime's gtap_thread.cuh and against this
// repository's include/gtap_thread.cuh.
//
//   cilksort_lowered N [REPS]   sorts N std::mt19937(42) keys in place,
//                               checks against std::sort, prints one JSON line
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <algorithm>
#include <climits>
#include <random>
#include <vector>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

#define TASK_SPAWN_CUTOFF_SORT 64
#define TASK_SPAWN_CUTOFF_MERGE 256

struct SortFrame {
    int* arr;
    int* tmp;
    int n;
    int pad;
};
struct MergeFrame {
    int* a;
    int* b;
    int* dst;
    int a_len;
    int b_len;
};
const size_t __gtap_auto_task_data_size = sizeof(SortFrame) > sizeof(MergeFrame) ? sizeof(SortFrame) : sizeof(MergeFrame);

// L1-bypassing load: keys are written by tasks on other SMs
__device__ __forceinline__ int key_load(const int* p) {
    int v;
    asm volatile("ld.global.cg.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// cilksort.cu:17-36
__device__ __forceinline__ void merge_device(const int* a, int a_len, const int* b, int b_len, int* dst) {
    int i = 0, j = 0, t = 0;
    while (i < a_len && j < b_len) {
        const int av = key_load(a + i), bv = key_load(b + j);
        if (av < bv) {
            dst[t++] = av;
            ++i;
        } else {
            dst[t++] = bv;
            ++j;
        }
    }
    while (i < a_len) dst[t++] = key_load(a + i++);
    while (j < b_len) dst[t++] = key_load(b + j++);
}

// cilksort.cu:38-49: largest index with x[index] <= val
__device__ __forceinline__ int binary_search_device(const int* x, int len, int val) {
    int low = -1, high = len;
    while (low + 1 < high) {
        const int mid = (low + high) / 2;
        if (key_load(x + mid) <= val) low = mid;
        else high = mid;
    }
    return low;
}

// cilksort.cu:51-86: bitonic network over TASK_SPAWN_CUTOFF_SORT keys padded with INT_MAX
__device__ __forceinline__ void sort_small_device(int* arr, int n) {
    int buf[TASK_SPAWN_CUTOFF_SORT];
#pragma unroll
    for (int i = 0; i < TASK_SPAWN_CUTOFF_SORT; ++i) buf[i] = i < n ? key_load(arr + i) : INT_MAX;
    for (int k = 2; k <= TASK_SPAWN_CUTOFF_SORT; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (int i = 0; i < TASK_SPAWN_CUTOFF_SORT; ++i) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const int x = buf[i], y = buf[ixj];
                    if (up ? (x > y) : (x < y)) {
                        buf[i] = y;
                        buf[ixj] = x;
                    }
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < TASK_SPAWN_CUTOFF_SORT; ++i)
        if (i < n) arr[i] = buf[i];
}

__device__ void cilkmerge_task(void* frame, int tid, TaskContext* ctx) {
    MergeFrame* f = (MergeFrame*)frame;
    switch (__gtap_get_task_state(tid)) {
        case 0: {
            int* a = f->a;
            int* b = f->b;
            int a_len = f->a_len, b_len = f->b_len;
            int* dst = f->dst;
            if (a_len < b_len) {
                int* t = a;
                a = b;
                b = t;
                const int tl = a_len;
                a_len = b_len;
                b_len = tl;
            }
            if (b_len == 0) {
                for (int i = 0; i < a_len; ++i) dst[i] = key_load(a + i);
                __threadfence();
                __gtap_finish_task(tid, ctx);
                return;
            }
            if (a_len + b_len < TASK_SPAWN_CUTOFF_MERGE) {
                merge_device(a, a_len, b, b_len, dst);
                __gtap_finish_task(tid, ctx);
                return;
            }
            const int a_split = (a_len + 1) / 2;
            const int b_split = binary_search_device(b, b_len, key_load(a + a_split - 1)) + 1;
            int child_count = 0;
            MergeFrame* c1 = (MergeFrame*)__gtap_spawn_task(ctx, tid, &child_count, cilkmerge_task, 0, nullptr, false);
            c1->a = a;
            c1->a_len = a_split;
            c1->b = b;
            c1->b_len = b_split;
            c1->dst = dst;
            MergeFrame* c2 = (MergeFrame*)__gtap_spawn_task(ctx, tid, &child_count, cilkmerge_task, 0, nullptr, false);
            c2->a = a + a_split;
            c2->a_len = a_len - a_split;
            c2->b = b + b_split;
            c2->b_len = b_len - b_split;
            c2->dst = dst + a_split + b_split;
            if (__gtap_set_state_for_join(tid, child_count, 1, 0)) return;
        }
        // fallthrough
        default:
            __gtap_finish_task(tid, ctx);
            return;
    }
}

__device__ __forceinline__ void spawn_merge(TaskContext* ctx, int tid, int* cc, int* a, int a_len, int* b, int b_len,
                                            int* dst) {
    MergeFrame* m = (MergeFrame*)__gtap_spawn_task(ctx, tid, cc, cilkmerge_task, 0, nullptr, false);
    m->a = a;
    m->a_len = a_len;
    m->b = b;
    m->b_len = b_len;
    m->dst = dst;
}

__device__ void cilksort_task(void* frame, int tid, TaskContext* ctx);

__device__ __forceinline__ void spawn_sort(TaskContext* ctx, int tid, int* cc, int* arr, int n, int* tmp) {
    SortFrame* s = (SortFrame*)__gtap_spawn_task(ctx, tid, cc, cilksort_task, 0, nullptr, false);
    s->arr = arr;
    s->n = n;
    s->tmp = tmp;
}

__device__ void cilksort_task(void* frame, int tid, TaskContext* ctx) {
    SortFrame* f = (SortFrame*)frame;
    int* arr = f->arr;
    int* tmp = f->tmp;
    const int n = f->n;
    const int len12 = n / 2, len1 = len12 / 2, len2 = len12 - len1;
    const int len34 = n - len12, len3 = len34 / 2, len4 = len34 - len3;
    int child_count = 0;
    switch (__gtap_get_task_state(tid)) {
        case 0:
            if (n < TASK_SPAWN_CUTOFF_SORT) {
                sort_small_device(arr, n);
                __gtap_finish_task(tid, ctx);
                return;
            }
            spawn_sort(ctx, tid, &child_count, arr, len1, tmp);
            spawn_sort(ctx, tid, &child_count, arr + len1, len2, tmp + len1);
            spawn_sort(ctx, tid, &child_count, arr + len12, len3, tmp + len12);
            spawn_sort(ctx, tid, &child_count, arr + len12 + len3, len4, tmp + len12 + len3);
            if (__gtap_set_state_for_join(tid, child_count, 1, 0)) return;
        // fallthrough
        case 1:
            child_count = 0;
            spawn_merge(ctx, tid, &child_count, arr, len1, arr + len1, len2, tmp);
            spawn_merge(ctx, tid, &child_count, arr + len12, len3, arr + len12 + len3, len4, tmp + len12);
            if (__gtap_set_state_for_join(tid, child_count, 2, 0)) return;
        // fallthrough
        case 2:
            child_count = 0;
            spawn_merge(ctx, tid, &child_count, tmp, len12, tmp + len12, len34, arr);
            if (__gtap_set_state_for_join(tid, child_count, 3, 0)) return;
        // fallthrough
        default:
            __gtap_finish_task(tid, ctx);
            return;
    }
}

__global__ void exec_kernel(int* data, int* buf, int n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        __gtap_push_initial_task(cilksort_task, 0);
        SortFrame* f = (SortFrame*)__gtap_get_task_data(0);
        f->arr = data;
        f->tmp = buf;
        f->n = n;
    }
    __gtap_execute_task_loop_device();
}

int main(int argc, char** argv) {
    const long long n = argc > 1 ? atoll(argv[1]) : (1ll << 24);
    const int reps = argc > 2 ? atoi(argv[2]) : 3;
    std::mt19937 rng(42);
    std::vector<int> h(n);
    for (long long i = 0; i < n; ++i) h[i] = (int)rng();
    std::vector<int> gold = h;
    std::sort(gold.begin(), gold.end());
    cudaError_t err = gtap_initialize();
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
        printf("{\"error\": \"%s\"}\n", cudaGetErrorString(err));
        return 1;
    }
    int* d_data = nullptr;
    int* d_buf = nullptr;
    if (cudaMalloc(&d_data, sizeof(int) * n) != cudaSuccess || cudaMalloc(&d_buf, sizeof(int) * n) != cudaSuccess) return 1;
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    bool ok = true;
    printf("{\"program\": \"cilksort\", \"n\": %lld, \"grid\": %d, \"block\": %d, \"ms\": [", n, GTAP_GRID_SIZE,
           GTAP_BLOCK_SIZE);
    std::vector<int> out(n);
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        cudaMemcpy(d_data, h.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
        cudaEventRecord(start);
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(d_data, d_buf, (int)n);
        cudaEventRecord(stop);
        if (gtap_synchronize() != cudaSuccess) return 1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, start, stop);
        cudaMemcpy(out.data(), d_data, sizeof(int) * n, cudaMemcpyDeviceToHost);
        ok = ok && out == gold;
        printf("%s%.4f", r ? ", " : "", ms);
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("], \"sorted\": %s, \"error_code\": %d}\n", ok ? "true" : "false", code);
    cudaFree(d_data);
    cudaFree(d_buf);
    gtap_finalize();
    return (code != 0 || !ok) ? 1 : 0;
}
