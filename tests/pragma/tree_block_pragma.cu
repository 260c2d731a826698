// tree_block_pragma.cu -- a complete binary tree in block mode written with the
// gtap pragmas in the shape of the reference's block binary tree: the taskwait
// sits in the else branch, thread 0 forks both children with their results
// assigned, the block waits, then every thread takes a share of the node's own
// work and the node returns its value plus its children's.
//
//   tree HEIGHT WORK   prints one JSON line
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_block.cuh"

__device__ unsigned long long d_result;

__device__ unsigned long long node_value(int node, int work) {
    __shared__ unsigned long long acc;
    if (threadIdx.x == 0) acc = 0;
    __syncthreads();
    unsigned long long part = 0;
    for (int i = threadIdx.x; i < work; i += blockDim.x)
        part += ((unsigned)node * 2654435761u + (unsigned)i * 40503u) >> 22;
    atomicAdd(&acc, part);
    __syncthreads();
    const unsigned long long v = acc;
    __syncthreads();
    return v;
}

#pragma gtap function
__device__ unsigned long long tree(int node, int height, int work) {
    unsigned long long l = 0, r = 0;
    if (height == 0) {
        return node_value(node, work);
    } else {
        if (threadIdx.x == 0) {
            int lc = 2 * node + 1;
            int rc = 2 * node + 2;
            #pragma gtap task
            l = tree(lc, height - 1, work);
            #pragma gtap task
            r = tree(rc, height - 1, work);
        }
        #pragma gtap taskwait
        unsigned long long own = node_value(node, work);
        return own + l + r;
    }
}

__global__ void exec_kernel(int height, int work) {
    #pragma gtap entry
    d_result = tree(0, height, work);
}

int main(int argc, char** argv) {
    const int height = argc > 1 ? atoi(argv[1]) : 10;
    const int work = argc > 2 ? atoi(argv[2]) : 300;
    if (gtap_initialize() != cudaSuccess) return 1;
    exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(height, work);
    if (gtap_synchronize() != cudaSuccess) return 1;
    unsigned long long result = 0;
    cudaMemcpyFromSymbol(&result, d_result, sizeof(result));
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("{\"program\": \"tree_block_pragma\", \"height\": %d, \"work\": %d, \"result\": %llu, \"error_code\": %d}\n",
           height, work, result, code);
    gtap_finalize();
    return code != 0;
}
