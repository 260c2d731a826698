// nq_lowered.cu -- evaluation/2-comparison/nq/gtap_nq.cu:10-60 (the
// no-taskwait build, -DGTAP_ASSUME_NO_TASKWAIT) hand-lowered to the
// reference's task ABI: a task per placed row, rows deeper than the cutoff
// searched serially, every solution counted with an atomicAdd.  Compiles
// against the reference runtime's gtap_thread.cuh and against this
// repository's include/gtap_thread.cuh.
//
//   nq_lowered N [CUTOFF_DEPTH] [REPS]   prints one JSON line
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

struct NqFrame {
    int row;
    uint32_t column;
    uint32_t left;
    uint32_t down;
    uint32_t right;
};
const size_t __gtap_auto_task_data_size = sizeof(NqFrame);

__device__ int d_answer;
__device__ int d_grid_size;
__device__ int d_cutoff_depth;

// gtap_nq.cu:10-23 serial_search: the same depth-first search over the rows
// below `row`, as a loop (one placed column per row kept in a byte array, the
// masks rebuilt when a placement is undone), one atomicAdd per solution
__device__ __noinline__ void serial_search(int row, uint32_t column, uint32_t left, uint32_t down, uint32_t right) {
    const int n = d_grid_size;
    if (row == n) {
        atomicAdd(&d_answer, 1);
        return;
    }
    const uint32_t mask = (n < 32 ? (1u << n) - 1 : 0xFFFFFFFFu);
    unsigned long long L = left, R = (unsigned long long)right << 32;
    uint32_t C = column;
    unsigned char chosen[32];
    int d = 0;
    const int last = n - row - 1;
    uint32_t avail = mask & ~(C | (uint32_t)L | (uint32_t)(R >> 32));
    for (;;) {
        if (avail) {
            const uint32_t p = avail & (0u - avail);
            avail &= avail - 1;
            if (d == last) {
                atomicAdd(&d_answer, 1);
                continue;
            }
            chosen[d] = (unsigned char)(__ffs((int)p) - 1);
            C |= p;
            L = (L | p) << 1;
            R = (R | ((unsigned long long)p << 32)) >> 1;
            ++d;
            avail = mask & ~(C | (uint32_t)L | (uint32_t)(R >> 32));
            continue;
        }
        if (d == 0) break;
        --d;
        const uint32_t p = 1u << chosen[d];
        C &= ~p;
        L = (L >> 1) & ~(unsigned long long)p;
        R = (R << 1) & ~((unsigned long long)p << 32);
        avail = mask & ~(C | (uint32_t)L | (uint32_t)(R >> 32)) & ~((p << 1) - 1u);
    }
    (void)down;
}

__device__ void nq_task(void* frame, int tid, TaskContext* ctx) {
    const NqFrame f = *(const NqFrame*)frame;
    const int grid_size = d_grid_size;
    if (f.row > d_cutoff_depth) {
        serial_search(f.row, f.column, f.left, f.down, f.right);
        __gtap_finish_task(tid, ctx);
        return;
    }
    const uint32_t mask = (grid_size < 32 ? (1u << grid_size) - 1 : 0xFFFFFFFFu);
    uint32_t avail = mask & ~(f.column | f.left | f.right);
    int child_count = 0;
    while (avail) {
        const uint32_t p = avail & (0u - avail);
        avail -= p;
        NqFrame* c = (NqFrame*)__gtap_spawn_task(ctx, tid, &child_count, nq_task, 0, nullptr, false);
        c->row = f.row + 1;
        c->column = f.column | p;
        c->left = (f.left | p) << 1;
        c->down = f.down | p;
        c->right = (f.right | p) >> 1;
    }
    __gtap_finish_task(tid, ctx);
}

__global__ void exec_kernel() {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        __gtap_push_initial_task(nq_task, 0);
        NqFrame* f = (NqFrame*)__gtap_get_task_data(0);
        f->row = 0;
        f->column = f->left = f->down = f->right = 0;
    }
    __gtap_execute_task_loop_device();
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 13;
    const int cutoff = argc > 2 ? atoi(argv[2]) : 7;
    const int reps = argc > 3 ? atoi(argv[3]) : 5;
    cudaMemcpyToSymbol(d_grid_size, &n, sizeof(int));
    cudaMemcpyToSymbol(d_cutoff_depth, &cutoff, sizeof(int));
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
    printf("{\"program\": \"nq\", \"n\": %d, \"cutoff\": %d, \"grid\": %d, \"block\": %d, \"ms\": [", n, cutoff,
           GTAP_GRID_SIZE, GTAP_BLOCK_SIZE);
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        const int zero = 0;
        cudaMemcpyToSymbol(d_answer, &zero, sizeof(int));
        cudaEventRecord(start);
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>();
        cudaEventRecord(stop);
        if (gtap_synchronize() != cudaSuccess) return 1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, start, stop);
        cudaMemcpyFromSymbol(&result, d_answer, sizeof(int));
        printf("%s%.4f", r ? ", " : "", ms);
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("], \"result\": %d, \"error_code\": %d}\n", result, code);
    gtap_finalize();
    return code != 0;
}
