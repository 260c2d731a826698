// nq_pragma.cu -- n-queens written with the gtap pragmas: one task per row up
// to the cutoff depth, a serial search below it, solutions counted with an
// atomic (no taskwait: build with -DGTAP_ASSUME_NO_TASKWAIT).
//
//   nq N CUTOFF   prints one JSON line
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

__device__ unsigned long long d_count;

__device__ int nq_serial(int n, int row, unsigned cols, unsigned left, unsigned right) {
    if (row == n) return 1;
    int total = 0;
    unsigned avail = ((1u << n) - 1u) & ~(cols | left | right);
    while (avail) {
        const unsigned p = avail & (0u - avail);
        avail -= p;
        total += nq_serial(n, row + 1, cols | p, (left | p) << 1, (right | p) >> 1);
    }
    return total;
}

#pragma gtap function
__device__ void nq(int n, int cutoff, int row, unsigned cols, unsigned left, unsigned right) {
    if (row > cutoff || row == n) {
        atomicAdd(&d_count, (unsigned long long)nq_serial(n, row, cols, left, right));
        return;
    }
    unsigned avail = ((1u << n) - 1u) & ~(cols | left | right);
    while (avail) {
        const unsigned p = avail & (0u - avail);
        avail -= p;
        #pragma gtap task
        nq(n, cutoff, row + 1, cols | p, (left | p) << 1, (right | p) >> 1);
    }
}

__global__ void exec_kernel(int n, int cutoff) {
    #pragma gtap entry
    nq(n, cutoff, 0, 0u, 0u, 0u);
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 10;
    const int cutoff = argc > 2 ? atoi(argv[2]) : n - 1;
    if (gtap_initialize() != cudaSuccess) return 1;
    const unsigned long long zero = 0;
    cudaMemcpyToSymbol(d_count, &zero, sizeof(zero));
    exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(n, cutoff);
    if (gtap_synchronize() != cudaSuccess) return 1;
    unsigned long long count = 0;
    cudaMemcpyFromSymbol(&count, d_count, sizeof(count));
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("{\"program\": \"nq_pragma\", \"n\": %d, \"result\": %llu, \"error_code\": %d}\n", n, count, code);
    gtap_finalize();
    return code != 0;
}
