// cilksort_pragma.cu -- a four-way mergesort written with the gtap pragmas:
// void tasks, three taskwaits, locals that live across them, and a parallel
// merge that splits at a binary search.
//
//   cilksort N SEED   prints one JSON line (sorted: whether the output is ascending
//                     and a permutation of the input, by a key sum and xor)
#include <stdio.h>
#include <stdlib.h>
#include <vector>
#include <cuda_runtime.h>

#include "gtap_thread.cuh"

#define SORT_CUTOFF 64
#define MERGE_CUTOFF 256

__device__ void seq_merge(const int* a, int na, const int* b, int nb, int* dst) {
    int i = 0, j = 0, k = 0;
    while (i < na && j < nb) dst[k++] = (a[i] <= b[j]) ? a[i++] : b[j++];
    while (i < na) dst[k++] = a[i++];
    while (j < nb) dst[k++] = b[j++];
}

__device__ void insertion_sort(int* a, int n) {
    for (int i = 1; i < n; ++i) {
        const int v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) {
            a[j + 1] = a[j];
            --j;
        }
        a[j + 1] = v;
    }
}

// number of keys of b[0..nb) that are <= v
__device__ int upper(const int* b, int nb, int v) {
    int lo = 0, hi = nb;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (b[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

#pragma gtap function
__device__ void pmerge(const int* a, int na, const int* b, int nb, int* dst) {
    if (na < nb) {
        const int* t = a;
        a = b;
        b = t;
        int tn = na;
        na = nb;
        nb = tn;
    }
    if (na + nb < MERGE_CUTOFF || nb == 0) {
        seq_merge(a, na, b, nb, dst);
        return;
    }
    int sa = (na + 1) / 2;
    int sb = upper(b, nb, a[sa - 1]);
    #pragma gtap task
    pmerge(a, sa, b, sb, dst);
    #pragma gtap task
    pmerge(a + sa, na - sa, b + sb, nb - sb, dst + sa + sb);
    #pragma gtap taskwait
}

#pragma gtap function
__device__ void csort(int* arr, int* tmp, int n) {
    if (n < SORT_CUTOFF) {
        insertion_sort(arr, n);
        return;
    }
    int h = n / 2;
    int q1 = h / 2;
    int q3 = (n - h) / 2;
    #pragma gtap task
    csort(arr, tmp, q1);
    #pragma gtap task
    csort(arr + q1, tmp + q1, h - q1);
    #pragma gtap task
    csort(arr + h, tmp + h, q3);
    #pragma gtap task
    csort(arr + h + q3, tmp + h + q3, n - h - q3);
    #pragma gtap taskwait
    #pragma gtap task
    pmerge(arr, q1, arr + q1, h - q1, tmp);
    #pragma gtap task
    pmerge(arr + h, q3, arr + h + q3, n - h - q3, tmp + h);
    #pragma gtap taskwait
    #pragma gtap task
    pmerge(tmp, h, tmp + h, n - h, arr);
    #pragma gtap taskwait
}

__global__ void exec_kernel(int* arr, int* tmp, int n) {
    #pragma gtap entry
    csort(arr, tmp, n);
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 100000;
    const unsigned seed = argc > 2 ? (unsigned)atoi(argv[2]) : 1;
    std::vector<int> keys(n);
    unsigned s = seed;
    long long sum = 0;
    int x = 0;
    for (int i = 0; i < n; ++i) {
        s = s * 1664525u + 1013904223u;
        keys[i] = (int)(s >> 1) - (1 << 30);
        sum += keys[i];
        x ^= keys[i];
    }
    int *d_arr, *d_tmp;
    cudaMalloc(&d_arr, sizeof(int) * n);
    cudaMalloc(&d_tmp, sizeof(int) * n);
    cudaMemcpy(d_arr, keys.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (gtap_initialize() != cudaSuccess) return 1;
    exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(d_arr, d_tmp, n);
    if (gtap_synchronize() != cudaSuccess) return 1;
    cudaMemcpy(keys.data(), d_arr, sizeof(int) * n, cudaMemcpyDeviceToHost);
    bool ok = true;
    long long sum2 = 0;
    int x2 = 0;
    for (int i = 0; i < n; ++i) {
        if (i && keys[i - 1] > keys[i]) ok = false;
        sum2 += keys[i];
        x2 ^= keys[i];
    }
    int code = 0;
    gtap_get_runtime_error_code(&code);
    printf("{\"program\": \"cilksort_pragma\", \"n\": %d, \"sorted\": %s, \"error_code\": %d}\n", n,
           (ok && sum == sum2 && x == x2) ? "true" : "false", code);
    gtap_finalize();
    return code != 0;
}
