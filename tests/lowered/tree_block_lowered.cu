// tree_block_lowered.cu -- a complete binary tree in the shape of
// examples/binary_tree/binary_tree_block.cu:85-113 (1 block = 1 task: thread
// 0 forks both children, the block waits, then every thread does the node's
// own work), with integer work so the result is exact: each node's value is a
// block-wide sum over its work items, and a node returns its own value plus
// its children's results, read from their retained frames after the
// taskwait.  Written by hand in the form of the reference's block-mode task
// ABI; compiles against include/gtap_block.cuh.
//
//   tree_block_lowered HEIGHT WORK REPS   prints one JSON line
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_block.cuh"

struct TreeFrame {
    int node;
    int height;
    int c0;   // child task ids (retained until read)
    int c1;
    unsigned long long ret;
};
struct EntryFrame {
    int height;
    int c0;
    int pad0;
    int pad1;
};
const size_t __gtap_auto_task_data_size = sizeof(TreeFrame) > sizeof(EntryFrame) ? sizeof(TreeFrame) : sizeof(EntryFrame);

__device__ int d_work;
__device__ unsigned long long d_result;

// Every thread of the block takes a share of the node's work items; the
// block's sum is returned to every thread.
__device__ unsigned long long node_value(int node) {
    __shared__ unsigned long long acc;
    if (threadIdx.x == 0) acc = 0;
    __syncthreads();
    unsigned long long part = 0;
    for (int i = threadIdx.x; i < d_work; i += blockDim.x)
        part += ((unsigned)node * 2654435761u + (unsigned)i * 40503u) >> 22;
    atomicAdd(&acc, part);
    __syncthreads();
    const unsigned long long v = acc;
    __syncthreads();
    return v;
}

__device__ void tree_task(void* frame, int tid, TaskContext* ctx) {
    TreeFrame* f = (TreeFrame*)frame;
    switch (__gtap_get_task_state(tid)) {
        case 0: {
            if (f->height == 0) {
                const unsigned long long own = node_value(f->node);
                if (threadIdx.x == 0) f->ret = own;
                __gtap_finish_task(tid, ctx);
                return;
            }
            if (threadIdx.x == 0) {
                int child_count = 0;
                TreeFrame* l = (TreeFrame*)__gtap_spawn_task(ctx, tid, &child_count, tree_task, 0, &f->c0, true);
                l->node = 2 * f->node + 1;
                l->height = f->height - 1;
                TreeFrame* r = (TreeFrame*)__gtap_spawn_task(ctx, tid, &child_count, tree_task, 0, &f->c1, true);
                r->node = 2 * f->node + 2;
                r->height = f->height - 1;
            }
            if (__gtap_set_state_for_join_block(tid, ctx, 1, 0)) return;
        }
        // fallthrough
        case 1: {
            const unsigned long long own = node_value(f->node);
            if (threadIdx.x == 0) {
                const unsigned long long a = ((TreeFrame*)__gtap_get_task_data(f->c0))->ret;
                const unsigned long long b = ((TreeFrame*)__gtap_get_task_data(f->c1))->ret;
                __gtap_release_task_id(f->c0);
                __gtap_release_task_id(f->c1);
                f->ret = own + a + b;
            }
            __gtap_finish_task(tid, ctx);
            return;
        }
        default:
            __gtap_finish_task(tid, ctx);
            return;
    }
}

// #pragma gtap entry: d_result = tree(0, height)
__device__ void entry_task(void* frame, int tid, TaskContext* ctx) {
    EntryFrame* e = (EntryFrame*)frame;
    switch (__gtap_get_task_state(tid)) {
        case 0: {
            if (threadIdx.x == 0) {
                int child_count = 0;
                TreeFrame* c = (TreeFrame*)__gtap_spawn_task(ctx, tid, &child_count, tree_task, 0, &e->c0, true);
                c->node = 0;
                c->height = e->height;
            }
            if (__gtap_set_state_for_join_block(tid, ctx, 1, 0)) return;
        }
        // fallthrough
        case 1:
            if (threadIdx.x == 0) {
                d_result = ((TreeFrame*)__gtap_get_task_data(e->c0))->ret;
                __gtap_release_task_id(e->c0);
            }
            __gtap_finish_task(tid, ctx);
            return;
        default:
            __gtap_finish_task(tid, ctx);
            return;
    }
}

__global__ void exec_kernel(int height) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        __gtap_push_initial_task(entry_task, 0);
        ((EntryFrame*)__gtap_get_task_data(0))->height = height;
    }
    __gtap_execute_task_loop_device();
}

int main(int argc, char** argv) {
    const int height = argc > 1 ? atoi(argv[1]) : 12;
    const int work = argc > 2 ? atoi(argv[2]) : 512;
    const int reps = argc > 3 ? atoi(argv[3]) : 3;
    if (cudaMemcpyToSymbol(d_work, &work, sizeof(int)) != cudaSuccess) return 1;
    cudaError_t err = gtap_initialize();
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
        printf("{\"error\": \"%s\"}\n", cudaGetErrorString(err));
        return 1;
    }
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    unsigned long long result = 0;
    printf("{\"program\": \"tree_block\", \"height\": %d, \"work\": %d, \"grid\": %d, \"block\": %d, \"ms\": [", height,
           work, GTAP_GRID_SIZE, GTAP_BLOCK_SIZE);
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        cudaEventRecord(start);
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(height);
        cudaEventRecord(stop);
        err = gtap_synchronize();
        if (err != cudaSuccess) return 1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, start, stop);
        cudaMemcpyFromSymbol(&result, d_result, sizeof(result));
        printf("%s%.4f", r ? ", " : "", ms);
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("], \"result\": %llu, \"error_code\": %d}\n", result, code);
    gtap_finalize();
    return code != 0;
}
