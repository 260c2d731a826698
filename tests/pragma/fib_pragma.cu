// fib_pragma.cu -- fib(n) written with the gtap pragmas (the source form the
// reference's examples use), lowered by gtap_b200.lower before nvcc.
//
//   fib N CUTOFF REPS   prints one JSON line (results and CUDA-event times of each launch)
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

__device__ int d_result;
__device__ int d_cutoff;

// below the cutoff: the same call tree as the recursion, walked with a bit
// set of pending arguments instead of a device stack
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

#pragma gtap function
__device__ int fib(int n) {
    if (n < 2) return n;
    if (n < d_cutoff) return fib_serial(n);
    int a, b;
    #pragma gtap task
    a = fib(n - 1);
    #pragma gtap task
    b = fib(n - 2);
    #pragma gtap taskwait
    return a + b;
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
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    int result = -1;
    printf("{\"program\": \"fib_pragma\", \"n\": %d, \"cutoff\": %d, \"grid\": %d, \"block\": %d, \"results\": [",
           n, cutoff, GTAP_GRID_SIZE, GTAP_BLOCK_SIZE);
    float ms[64];
    const int nt = reps < 64 ? reps : 64;
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        cudaEventRecord(start);
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(n);
        cudaEventRecord(stop);
        if (gtap_synchronize() != cudaSuccess) return 1;
        if (r < nt) cudaEventElapsedTime(&ms[r], start, stop);
        cudaMemcpyFromSymbol(&result, d_result, sizeof(int));
        printf("%s%d", r ? ", " : "", result);
    }
    printf("], \"ms\": [");
    for (int r = 0; r < nt; ++r) printf("%s%.4f", r ? ", " : "", ms[r]);
    printf("]");
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf(", \"error_code\": %d}\n", code);
    gtap_finalize();
    return code != 0;
}
