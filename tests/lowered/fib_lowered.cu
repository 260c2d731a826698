// fib_lowered.cu -- evaluation/2-comparison/fib/gtap_fib.cu:10-27 (and, with a
// cutoff, evaluation/3-epaq/fib/fib_queue_1.cu:9-26) written by hand in the
// form the reference's task ABI expects from clang-gtap: one switch state
// machine per `#pragma gtap function`, children's results read from their
// retained frames after the taskwait, and the entry as task 0.  The same file
// compiles against the reference runtime's runtime/gtap_thread.cuh and
// against this repository's include/gtap_thread.cuh.
//
//   fib_lowered N [CUTOFF] [REPS]   prints one JSON line
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

struct FibFrame {
    int n;
    int ret;   // result, read by the parent after its taskwait
    int c0;    // child task ids (retained until read)
    int c1;
};
struct EntryFrame {
    int n;
    int c0;
    int pad0;
    int pad1;
};
const size_t __gtap_auto_task_data_size = sizeof(FibFrame) > sizeof(EntryFrame) ? sizeof(FibFrame) : sizeof(EntryFrame);

__device__ int d_result;
__device__ int d_cutoff;

// fib_queue_1.cu:9-14 fib_sequential, as a loop over the same call tree (the
// pending n-1 calls form a strictly decreasing set, kept as bits)
__device__ __noinline__ int fib_serial(int n) {
    unsigned long long pending = 0;
    unsigned sum = 0;
    int m = n;
    for (;;) {
        if (m >= 2) {
            pending |= 1ull << (m - 1);
            m -= 2;
            continue;
        }
        sum += (unsigned)m;
        if (pending == 0) break;
        m = __ffsll((long long)pending) - 1;
        pending &= pending - 1;
    }
    return (int)sum;
}

__device__ void fib_task(void* frame, int tid, TaskContext* ctx) {
    FibFrame* f = (FibFrame*)frame;
    switch (__gtap_get_task_state(tid)) {
        case 0: {
            const int n = f->n;
            if (n < 2) {
                f->ret = n;
                __gtap_finish_task(tid, ctx);
                return;
            }
            if (n < d_cutoff) {
                f->ret = fib_serial(n);
                __gtap_finish_task(tid, ctx);
                return;
            }
            int child_count = 0;
            FibFrame* a = (FibFrame*)__gtap_spawn_task(ctx, tid, &child_count, fib_task, 0, &f->c0, true);
            a->n = n - 1;
            FibFrame* b = (FibFrame*)__gtap_spawn_task(ctx, tid, &child_count, fib_task, 0, &f->c1, true);
            b->n = n - 2;
            if (__gtap_set_state_for_join(tid, child_count, 1, 0)) return;
        }
        // fallthrough
        case 1: {
            const int a = ((FibFrame*)__gtap_get_task_data(f->c0))->ret;
            const int b = ((FibFrame*)__gtap_get_task_data(f->c1))->ret;
            __gtap_release_task_id(f->c0);
            __gtap_release_task_id(f->c1);
            f->ret = a + b;
            __gtap_finish_task(tid, ctx);
            return;
        }
        default:
            __gtap_finish_task(tid, ctx);
            return;
    }
}

// #pragma gtap entry: d_result = fib(n)
__device__ void entry_task(void* frame, int tid, TaskContext* ctx) {
    EntryFrame* e = (EntryFrame*)frame;
    switch (__gtap_get_task_state(tid)) {
        case 0: {
            int child_count = 0;
            FibFrame* c = (FibFrame*)__gtap_spawn_task(ctx, tid, &child_count, fib_task, 0, &e->c0, true);
            c->n = e->n;
            if (__gtap_set_state_for_join(tid, child_count, 1, 0)) return;
        }
        // fallthrough
        case 1:
            d_result = ((FibFrame*)__gtap_get_task_data(e->c0))->ret;
            __gtap_release_task_id(e->c0);
            __gtap_finish_task(tid, ctx);
            return;
        default:
            __gtap_finish_task(tid, ctx);
            return;
    }
}

__global__ void exec_kernel(int n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        __gtap_push_initial_task(entry_task, 0);
        ((EntryFrame*)__gtap_get_task_data(0))->n = n;
    }
    __gtap_execute_task_loop_device();
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 30;
    const int cutoff = argc > 2 ? atoi(argv[2]) : 0;
    const int reps = argc > 3 ? atoi(argv[3]) : 5;
    if (cudaMemcpyToSymbol(d_cutoff, &cutoff, sizeof(int)) != cudaSuccess) return 1;
    cudaError_t err = gtap_initialize();
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
        printf("{\"error\": \"%s\"}\n", cudaGetErrorString(err));
        return 1;
    }
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    int result = -1;
    printf("{\"program\": \"fib\", \"n\": %d, \"cutoff\": %d, \"grid\": %d, \"block\": %d, \"ms\": [", n, cutoff,
           GTAP_GRID_SIZE, GTAP_BLOCK_SIZE);
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        cudaEventRecord(start);
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(n);
        cudaEventRecord(stop);
        err = gtap_synchronize();
        if (err != cudaSuccess) return 1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, start, stop);
        cudaMemcpyFromSymbol(&result, d_result, sizeof(int));
        printf("%s%.4f", r ? ", " : "", ms);
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("], \"result\": %d, \"error_code\": %d}\n", result, code);
    gtap_finalize();
    return code != 0;
}
