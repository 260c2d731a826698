// bfs_block_lowered.cu -- examples/asynchronous_bfs/asynchronous_bfs_block.cu:19-37
// written by hand in the form the reference's block-mode task ABI expects
// from clang-gtap (GTAP_ASSUME_NO_TASKWAIT, as its Makefile builds it): one
// task per vertex, every thread of the block strides over the adjacency list
// and spawns a task for each neighbour it improved.  Compiles against
// include/gtap_block.cuh.
//
//   bfs_block_lowered SCALE SEED REPS OUT   prints one JSON line; writes the
//                                          depth array (int32) to OUT
#include <stdio.h>
#include <stdlib.h>
#include <vector>
#include <cuda_runtime.h>

#include "gtap_block.cuh"

// R-MAT generator of libgtap_b200.so (declared here: gtap.h's host names
// clash with the reference host functions this program uses)
extern "C" int gtap_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed, int32_t* row, int32_t* col);

struct BfsFrame {
    int v;
};
const size_t __gtap_auto_task_data_size = sizeof(BfsFrame);

__device__ int* g_row;
__device__ int* g_col;
__device__ int* g_depth;

// asynchronous_bfs_block.cu:19-31
__device__ void bfs_task(void* frame, int tid, TaskContext* ctx) {
    const int v = ((BfsFrame*)frame)->v;
    const int dv = g_depth[v];
    const int row_start = g_row[v];
    const int row_end = g_row[v + 1];
    for (int e = row_start + threadIdx.x; e < row_end; e += blockDim.x) {
        const int u = g_col[e];
        const int old = atomicMin(&g_depth[u], dv + 1);
        if (old > dv + 1) {
            int child_count = 0;
            BfsFrame* c = (BfsFrame*)__gtap_spawn_task(ctx, tid, &child_count, bfs_task, 0, nullptr, false);
            c->v = u;
        }
    }
    __gtap_finish_task(tid, ctx);
}

// asynchronous_bfs_block.cu:33-37: depth[source] = 0, then the entry task
__global__ void exec_kernel(int source) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        g_depth[source] = 0;
        __gtap_push_initial_task(bfs_task, 0);
        ((BfsFrame*)__gtap_get_task_data(0))->v = source;
    }
    __gtap_execute_task_loop_device();
}

int main(int argc, char** argv) {
    const int scale = argc > 1 ? atoi(argv[1]) : 14;
    const unsigned long long seed = argc > 2 ? strtoull(argv[2], nullptr, 10) : 42;
    const int reps = argc > 3 ? atoi(argv[3]) : 2;
    const char* out = argc > 4 ? argv[4] : nullptr;
    const int nv = 1 << scale;
    std::vector<int> row(nv + 1), col((size_t)nv * 16);
    if (gtap_gen_rmat(scale, 16, seed, row.data(), col.data()) != 0) return 1;
    int source = 0;
    for (int v = 0; v < nv; ++v)
        if (row[v + 1] - row[v] > row[source + 1] - row[source]) source = v;
    int *d_row, *d_col, *d_depth;
    cudaMalloc(&d_row, sizeof(int) * (nv + 1));
    cudaMalloc(&d_col, sizeof(int) * col.size());
    cudaMalloc(&d_depth, sizeof(int) * nv);
    cudaMemcpy(d_row, row.data(), sizeof(int) * (nv + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(d_col, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice);
    cudaMemcpyToSymbol(g_row, &d_row, sizeof(int*));
    cudaMemcpyToSymbol(g_col, &d_col, sizeof(int*));
    cudaMemcpyToSymbol(g_depth, &d_depth, sizeof(int*));
    cudaError_t err = gtap_initialize();
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
        printf("{\"error\": \"%s\"}\n", cudaGetErrorString(err));
        return 1;
    }
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    printf("{\"program\": \"bfs_block\", \"scale\": %d, \"source\": %d, \"grid\": %d, \"block\": %d, \"ms\": [", scale,
           source, GTAP_GRID_SIZE, GTAP_BLOCK_SIZE);
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        cudaMemset(d_depth, 0x3f, sizeof(int) * nv);   // INF = 0x3f3f3f3f
        cudaEventRecord(start);
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(source);
        cudaEventRecord(stop);
        err = gtap_synchronize();
        if (err != cudaSuccess) return 1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, start, stop);
        printf("%s%.4f", r ? ", " : "", ms);
    }
    std::vector<int> depth(nv);
    cudaMemcpy(depth.data(), d_depth, sizeof(int) * nv, cudaMemcpyDeviceToHost);
    if (out) {
        FILE* f = fopen(out, "wb");
        if (!f || fwrite(depth.data(), sizeof(int), nv, f) != (size_t)nv) return 1;
        fclose(f);
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("], \"error_code\": %d}\n", code);
    gtap_finalize();
    return code != 0;
}
