// bary_block_pragma.cu -- the probabilistic B-ary tree in block mode, in the
// shape of the reference's gtap_block_tree_load_compute.cu: thread 0 draws
// and spawns a node's children (each of B candidates kept with probability
// 1 - d/D), the block waits, then every thread takes a strided share of the
// node's seeded double loads and fused multiply-adds; the partial sums are
// added in thread order and the xor-words combined into the node's 32-bit
// mix, which is added to a 64-bit sum.  Deterministic for a given block size.
//
//   bary_block D B MEM_OPS ITERS LOG2_INPUT SEED REPS   prints one JSON line
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include <cuda_runtime.h>

#include "gtap_block.cuh"

__device__ const double* g_input;
__device__ unsigned g_input_mask;
__device__ unsigned long long d_sum;
__device__ unsigned long long d_nodes;

// MurmurHash3's 32-bit finaliser
__host__ __device__ __forceinline__ unsigned fmix32(unsigned h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

__device__ unsigned node_work_block(unsigned node, int mem_ops, int iters) {
    __shared__ double s_part[512];
    __shared__ unsigned s_xr[512];
    __shared__ unsigned s_mix;
    const int T = blockDim.x, t = threadIdx.x;
    const unsigned seed = fmix32(node ^ 0x2545f491u);
    double part = 0.0;
    for (int m = t; m < mem_ops; m += T) part += g_input[fmix32(seed + (unsigned)m) & g_input_mask];
    double y = 0.0;
    unsigned xr = 0;
    for (int it = t; it < iters; it += T) {
        const double x = (double)fmix32(seed + (unsigned)it * 0x632be5abu);
        y = fma(x, 1.0000001192092896, y);
        const unsigned long long bits = (unsigned long long)__double_as_longlong(y);
        xr ^= (unsigned)bits ^ (unsigned)(bits >> 32);
    }
    s_part[t] = part;
    s_xr[t] = xr;
    __syncthreads();
    if (t == 0) {
        double acc = 0.0;
        unsigned x = 0;
        for (int i = 0; i < T; ++i) {
            acc += s_part[i];
            x ^= s_xr[i];
        }
        s_mix = ((seed ^ 0x9e3779b9u) + (unsigned)(int)acc) ^ x;
    }
    __syncthreads();
    const unsigned mix = s_mix;
    __syncthreads();
    return mix;
}

#pragma gtap function
__device__ void bary(unsigned node, int depth, int D, int B, int mem_ops, int iters) {
    if (depth < D) {
        if (threadIdx.x == 0) {
            unsigned s = fmix32(node ^ ((unsigned)depth * 0x9e3779b9u));
            for (int k = 0; k < B; ++k) {
                s = fmix32(s + (unsigned)k);
                if ((int)(s % (unsigned)D) < D - depth) {
                    #pragma gtap task
                    bary(node * (unsigned)B + (unsigned)(k + 1), depth + 1, D, B, mem_ops, iters);
                }
            }
        }
        #pragma gtap taskwait
    }
    const unsigned mix = node_work_block(node, mem_ops, iters);
    if (threadIdx.x == 0) {
        atomicAdd(&d_sum, (unsigned long long)mix);
        atomicAdd(&d_nodes, 1ull);
    }
}

__global__ void exec_kernel(int D, int B, int mem_ops, int iters) {
    #pragma gtap entry
    bary(0u, 0, D, B, mem_ops, iters);
}

int main(int argc, char** argv) {
    const int D = argc > 1 ? atoi(argv[1]) : 8;
    const int B = argc > 2 ? atoi(argv[2]) : 3;
    const int mem_ops = argc > 3 ? atoi(argv[3]) : 16;
    const int iters = argc > 4 ? atoi(argv[4]) : 32;
    const int log2n = argc > 5 ? atoi(argv[5]) : 16;
    const unsigned long long seed = argc > 6 ? strtoull(argv[6], nullptr, 10) : 7ull;
    const int reps = argc > 7 ? atoi(argv[7]) : 2;
    if (D < 0 || B < 1 || B > 64 || mem_ops < 0 || iters < 0 || log2n < 0 || log2n > 26) return 2;
    // splitmix64 (Steele, Lea, Flood 2014) mapped to doubles in [-1, 1)
    const size_t n = (size_t)1 << log2n;
    std::vector<double> h(n);
    unsigned long long x = seed;
    for (size_t i = 0; i < n; ++i) {
        x += 0x9e3779b97f4a7c15ull;
        unsigned long long z = x;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        h[i] = (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
    double* d_input = nullptr;
    if (cudaMalloc(&d_input, n * sizeof(double)) != cudaSuccess) return 1;
    cudaMemcpy(d_input, h.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    const unsigned mask = (unsigned)(n - 1);
    cudaMemcpyToSymbol(g_input, &d_input, sizeof(d_input));
    cudaMemcpyToSymbol(g_input_mask, &mask, sizeof(mask));
    if (gtap_initialize() != cudaSuccess) return 1;
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    unsigned long long sum = 0, nodes = 0;
    printf("{\"program\": \"bary_block_pragma\", \"D\": %d, \"B\": %d, \"threads\": %d, \"ms\": [", D, B,
           GTAP_BLOCK_SIZE);
    for (int r = 0; r < reps; ++r) {
        if (r > 0 && gtap_reset() != cudaSuccess) return 1;
        const unsigned long long zero = 0;
        cudaMemcpyToSymbol(d_sum, &zero, sizeof(zero));
        cudaMemcpyToSymbol(d_nodes, &zero, sizeof(zero));
        cudaEventRecord(start);
        exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(D, B, mem_ops, iters);
        cudaEventRecord(stop);
        if (gtap_synchronize() != cudaSuccess) return 1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, start, stop);
        printf("%s%.4f", r ? ", " : "", ms);
        cudaMemcpyFromSymbol(&sum, d_sum, sizeof(sum));
        cudaMemcpyFromSymbol(&nodes, d_nodes, sizeof(nodes));
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("], \"sum\": %llu, \"nodes\": %llu, \"error_code\": %d}\n", sum, nodes, code);
    gtap_finalize();
    cudaFree(d_input);
    return code != 0;
}
