// walk_pragma.cu -- a ternary walk written with the gtap pragmas to exercise
// the lowering's control flow: taskwaits inside if/else branches, a spawn
// whose result is assigned only on one path, a spawn whose result is dropped,
// a const local and a multi-name declaration that live across a taskwait, a
// local that is in scope at a resume point but not used after it, and a
// second taskwait at the top level.
//
//   walk DEPTH ID   prints one JSON line
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

__device__ unsigned long long d_result;

#pragma gtap function
__device__ unsigned long long walk(int depth, int id) {
    const int k = id % 3;
    unsigned long long a = 0, b = 0, own = id;
    int scale = depth * 7 + 1;
    if (depth == 0) return own * scale;
    if (k == 0) {
        #pragma gtap task
        a = walk(depth - 1, 3 * id + 1);
        #pragma gtap task
        b = walk(depth - 1, 3 * id + 2);
        #pragma gtap taskwait
        own += a - b;
    } else {
        int spare = id & 7;
        own += spare;
        if (k == 1) {
            #pragma gtap task
            a = walk(depth - 1, 3 * id + 1);
        }
        #pragma gtap task
        walk(depth - 1, 3 * id + 2);
        #pragma gtap taskwait
        own += 2 * a + k;
    }
    #pragma gtap task
    b = walk(depth / 2, id + 1);
    #pragma gtap taskwait
    return own * scale + b;
}

__global__ void exec_kernel(int depth, int id) {
    #pragma gtap entry
    d_result = walk(depth, id);
}

int main(int argc, char** argv) {
    const int depth = argc > 1 ? atoi(argv[1]) : 8;
    const int id = argc > 2 ? atoi(argv[2]) : 0;
    if (gtap_initialize() != cudaSuccess) return 1;
    exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(depth, id);
    if (gtap_synchronize() != cudaSuccess) return 1;
    unsigned long long result = 0;
    cudaMemcpyFromSymbol(&result, d_result, sizeof(result));
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("{\"program\": \"walk_pragma\", \"depth\": %d, \"id\": %d, \"result\": %llu, \"error_code\": %d}\n",
           depth, id, result, code);
    gtap_finalize();
    return code != 0;
}
