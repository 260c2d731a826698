// fib_queues_pragma.cu -- fib(n) with queue hints on its spawns and its
// taskwait (EPAQ, the reference's `queue(expr)` clause): the recursion spreads
// its tasks over queues 0 and 1 by the parity of n, and parents resume on
// queue 2.  Built with -DGTAP_NUM_QUEUES=3.
//
//   fib_queues N CUTOFF REPS   prints one JSON line
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

__device__ int d_result;
__device__ int d_cutoff;

__device__ __noinline__ int fib_loop(int n) {
    int a = 0, b = 1;
    for (int i = 0; i < n; ++i) {
        const int t = a + b;
        a = b;
        b = t;
    }
    return a;
}

#pragma gtap function
__device__ int fib(int n) {
    if (n < 2) return n;
    if (n < d_cutoff) return fib_loop(n);
    int x, y;
    #pragma gtap task queue((n - 1) & 1)
    x = fib(n - 1);
    #pragma gtap task queue(n & 1)
    y = fib(n - 2);
    #pragma gtap taskwait queue(2)
    return x + y;
}

__global__ void exec_kernel(int n) {
    #pragma gtap entry
    d_result = fib(n);
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 25;
    const int cutoff = argc > 2 ? atoi(argv[2]) : 0;
    const int reps = argc > 3 ? atoi(argv[3]) : 2;
    cudaMemcpyToSymbol(d_cutoff, &cutoff, sizeof(int));
    if (gtap_initialize() != cudaSuccess) return 1;
    int result = -1;
    printf("{\"program\": \"fib_queues_pragma\", \"n\": %d, \"queues\": %d, \"results\": [", n, GTAP_NUM_QUEUES);
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(n);
        if (gtap_synchronize() != cudaSuccess) return 1;
        cudaMemcpyFromSymbol(&result, d_result, sizeof(int));
        printf("%s%d", r ? ", " : "", result);
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("], \"error_code\": %d}\n", code);
    gtap_finalize();
    return code != 0;
}
