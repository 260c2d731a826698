// gtap_block_programs.cuh -- the built-in task bodies of block-cooperative
// mode: every thread of the block runs the body, so leaf work is done by the
// whole block (sorts and merges staged in shared memory, BFS adjacency
// strided over the threads); spawns and results come from thread 0 unless
// noted.  The spawn trees are those of the thread-mode programs, hence of the
// reference recursions cited there:
//   cilksort / cilkmerge   examples/cilksort/cilksort.cu:89-164
//   mergesort              examples/mergesort/mergesort.cu:34-50
//   fib                    evaluation/2-comparison/fib/gtap_fib.cu:10-22
//   n-queens               evaluation/2-comparison/nq/gtap_nq.cu:10-55
//   BFS (block variant)    examples/asynchronous_bfs/asynchronous_bfs_block.cu:19-31
//   tree sum               examples/binary_tree/binary_tree_thread.cu:63-114 (int64 sums)
#pragma once
#include "gtap_block_sched.cuh"

namespace gtap {
namespace bprog {

using prog::K_BFS;
using prog::K_CILKMERGE;
using prog::K_CILKSORT;
using prog::K_FIB;
using prog::K_MERGESORT;
using prog::K_NQ;
using prog::K_TREESUM;

constexpr int kLeafMax = 2048;             // keys one leaf sort or merge stages in shared memory
constexpr int kSmemInts = 2 * kLeafMax;    // dynamic shared memory of the block kernel (16 KB)

__device__ __forceinline__ void* ptr_of(int lo, int hi) {
    return reinterpret_cast<void*>((unsigned long long)(unsigned)lo | ((unsigned long long)(unsigned)hi << 32));
}

// Sort n (1..kLeafMax) keys from src into dst: a bitonic network over the
// next power of two in shared memory, padded with INT_MAX (the padding sorts
// behind every key, so the first n outputs are the keys in order).
__device__ void block_sort(const int* src, int* dst, int n, int* s) {
    const int nt = blockDim.x;
    int P = 2;
    while (P < n) P <<= 1;
    for (int i = threadIdx.x; i < P; i += nt) s[i] = i < n ? ld_data(src + i) : 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < (P >> 1); i += nt) {
                const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                const int hi = lo + j;
                const bool up = (lo & k) == 0;
                const int a = s[lo], b = s[hi];
                if ((a > b) == up && a != b) {
                    s[lo] = b;
                    s[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < n; i += nt) dst[i] = s[i];
}

// Merge sorted a[0..alen) and b[0..blen) (alen + blen <= kLeafMax) into dst:
// both staged in shared memory with coalesced loads, each thread merges one
// equal share of the output from its merge-path split, and the output leaves
// through shared memory with coalesced stores.
__device__ void block_merge(const int* a, int alen, const int* b, int blen, int* dst, int* s) {
    const int nt = blockDim.x;
    const int total = alen + blen;
    int* sa = s;
    int* sb = s + alen;
    int* so = s + kLeafMax;
    for (int i = threadIdx.x; i < alen; i += nt) sa[i] = ld_data(a + i);
    for (int i = threadIdx.x; i < blen; i += nt) sb[i] = ld_data(b + i);
    __syncthreads();
    const int per = (total + nt - 1) / nt;
    const int d0 = min((int)threadIdx.x * per, total);
    const int d1 = min(d0 + per, total);
    // split of diagonal d0: i keys from a, d0 - i from b, a first on ties
    int lo = max(0, d0 - blen), hi = min(d0, alen);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (sa[mid] <= sb[d0 - mid - 1]) lo = mid + 1;
        else hi = mid;
    }
    int i = lo, j = d0 - lo;
    for (int k = d0; k < d1; ++k) {
        if (j >= blen || (i < alen && sa[i] <= sb[j])) so[k] = sa[i++];
        else so[k] = sb[j++];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += nt) dst[k] = so[k];
}

// dst[0..n) = a[0..n), any n.
__device__ void block_copy(const int* a, int n, int* dst) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = ld_data(a + i);
}

// Number of keys of sorted b[0..blen) that are <= val (cilksort.cu:38-49's
// binary search + 1).  Every round each thread reads one sample, so the range
// shrinks by a factor blockDim + 1 per round: three rounds for 2^24 keys.
__device__ int block_upper_bound(const int* b, int blen, int val) {
    const int nt = blockDim.x;
    int lo = 0, hi = blen;   // the count lies in [lo, hi]
    while (hi - lo > nt) {
        const int L = hi - lo;
        const int step = (L + nt) / (nt + 1);   // ceil(L / (nt + 1)) >= 1
        const int p = lo + ((int)threadIdx.x + 1) * step - 1;
        const bool le = p < hi && ld_data(b + p) <= val;
        const int c = __syncthreads_count(le);
        const int nlo = lo + c * step;
        hi = min(hi, lo + (c + 1) * step - 1);
        lo = nlo;
    }
    const int p = lo + (int)threadIdx.x;
    const bool le = p < hi && ld_data(b + p) <= val;
    return lo + __syncthreads_count(le);
}

__device__ __forceinline__ void spawn_merge(const Arena& A, BlockShared& S, const int* a, int alen, const int* b,
                                            int blen, int* dst) {
    prog::MergeFrame* m = reinterpret_cast<prog::MergeFrame*>(bt_spawn(A, S, K_CILKMERGE, nullptr, nullptr, false, false));
    m->a = a;
    m->b = b;
    m->dst = dst;
    m->alen = alen;
    m->blen = blen;
}

__device__ __forceinline__ void spawn_sort(const Arena& A, BlockShared& S, int* arr, int* tmp, const int* src, int n) {
    prog::SortFrame* c = reinterpret_cast<prog::SortFrame*>(bt_spawn(A, S, K_CILKSORT, nullptr, nullptr, false, false));
    c->arr = arr;
    c->tmp = tmp;
    c->src = src;
    c->n = n;
}

// cilksort.cu:89-125.  Leaves (a copy, or a merge below the cutoff) are done
// by the whole block; the split point comes from the block-wide search.
__device__ void cilkmerge_task(const Arena& A, BlockShared& S, int* smem) {
    if (bt_state(S) != 0) {   // resumed after the taskwait: nothing left to do
        bt_finish(S);
        return;
    }
    const int4 w0 = S.w0, w1 = S.w1;
    const int* a = reinterpret_cast<const int*>(ptr_of(w0.x, w0.y));
    const int* b = reinterpret_cast<const int*>(ptr_of(w0.z, w0.w));
    int* dst = reinterpret_cast<int*>(ptr_of(w1.x, w1.y));
    int alen = w1.z, blen = w1.w;
    if (alen < blen) {
        const int* t = a;
        a = b;
        b = t;
        const int tl = alen;
        alen = blen;
        blen = tl;
    }
    if (blen == 0) {
        block_copy(a, alen, dst);
        bt_finish(S);
        return;
    }
    if (alen + blen < bt_root(A, S).i1) {
        block_merge(a, alen, b, blen, dst, smem);
        bt_finish(S);
        return;
    }
    const int as = (alen + 1) / 2;
    const int bs = block_upper_bound(b, blen, ld_data(a + as - 1));
    if (threadIdx.x == 0) {
        spawn_merge(A, S, a, as, b, bs, dst);
        spawn_merge(A, S, a + as, alen - as, b + bs, blen - bs, dst + as + bs);
    }
    if (bt_join(A, S, 1, true)) return;
    bt_finish(S);
}

// cilksort.cu:127-164: four quarter sorts, two merges, one merge.  Leaves sort
// src into arr (so repeated runs read pristine input).
__device__ void cilksort_task(const Arena& A, BlockShared& S, int* smem) {
    const int4 w0 = S.w0, w1 = S.w1;
    int* arr = reinterpret_cast<int*>(ptr_of(w0.x, w0.y));
    int* tmp = reinterpret_cast<int*>(ptr_of(w0.z, w0.w));
    const int* src = reinterpret_cast<const int*>(ptr_of(w1.x, w1.y));
    const int n = w1.z;
    const int len12 = n / 2, len1 = len12 / 2, len2 = len12 - len1;
    const int len34 = n - len12, len3 = len34 / 2, len4 = len34 - len3;
    int st = bt_state(S);
    if (st == 0) {
        if (n < bt_root(A, S).i0) {
            if (n > 0) block_sort(src, arr, n, smem);
            bt_finish(S);
            return;
        }
        if (threadIdx.x == 0) {
            spawn_sort(A, S, arr, tmp, src, len1);
            spawn_sort(A, S, arr + len1, tmp + len1, src + len1, len2);
            spawn_sort(A, S, arr + len12, tmp + len12, src + len12, len3);
            spawn_sort(A, S, arr + len12 + len3, tmp + len12 + len3, src + len12 + len3, len4);
        }
        if (bt_join(A, S, 1)) return;
        st = 1;
    }
    if (st == 1) {
        if (threadIdx.x == 0) {
            spawn_merge(A, S, arr, len1, arr + len1, len2, tmp);
            spawn_merge(A, S, arr + len12, len3, arr + len12 + len3, len4, tmp + len12);
        }
        if (bt_join(A, S, 2)) return;
        st = 2;
    }
    if (st == 2) {
        if (threadIdx.x == 0) spawn_merge(A, S, tmp, len12, tmp + len12, len34, arr);
        if (bt_join(A, S, 3, true)) return;
        st = 3;
    }
    if (st != 3 && threadIdx.x == 0) GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.task, -1, st, 3);
    bt_finish(S);
}

// mergesort.cu:34-50: the halves sort into tmp (out as their scratch), then
// one cilkmerge of the halves into out.  Leaves sort in into out.
__device__ void mergesort_task(const Arena& A, BlockShared& S, int* smem) {
    const int4 w0 = S.w0, w1 = S.w1;
    const int* in = reinterpret_cast<const int*>(ptr_of(w0.x, w0.y));
    int* out = reinterpret_cast<int*>(ptr_of(w0.z, w0.w));
    int* tmp = reinterpret_cast<int*>(ptr_of(w1.x, w1.y));
    const int n = w1.z;
    const int nl = (n + 1) / 2;
    int st = bt_state(S);
    if (st == 0) {
        if (n <= bt_root(A, S).i0 || n <= 1) {
            if (n > 0) block_sort(in, out, n, smem);
            bt_finish(S);
            return;
        }
        if (threadIdx.x == 0) {
            prog::MsFrame* c1 = reinterpret_cast<prog::MsFrame*>(bt_spawn(A, S, K_MERGESORT, nullptr, nullptr, false, false));
            c1->in = in;
            c1->out = tmp;
            c1->tmp = out;
            c1->n = nl;
            prog::MsFrame* c2 = reinterpret_cast<prog::MsFrame*>(bt_spawn(A, S, K_MERGESORT, nullptr, nullptr, false, false));
            c2->in = in + nl;
            c2->out = tmp + nl;
            c2->tmp = out + nl;
            c2->n = n - nl;
        }
        if (bt_join(A, S, 1)) return;
        st = 1;
    }
    if (st == 1) {
        if (threadIdx.x == 0) spawn_merge(A, S, tmp, nl, tmp + nl, n - nl, out);
        if (bt_join(A, S, 2, true)) return;
        st = 2;
    }
    if (st != 2 && threadIdx.x == 0) GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.task, -1, st, 2);
    bt_finish(S);
}

// gtap_fib.cu:10-22 with fib_queue_1.cu's sequential cutoff; one block per task.
__device__ void fib_task(const Arena& A, BlockShared& S) {
    const int4 fr = S.w0;   // {n, a, b, slot}: the root's frame also carries thread mode's settings above the slot byte
    int st = bt_state(S);
    if (st == 0) {
        const int n = fr.x, cutoff = bt_root(A, S).i1;
        if (n < 2 || n < cutoff) {
            if (threadIdx.x == 0) bt_return_i32(A, S, fr.w & prog::kFibSlotMask, n < 2 ? n : prog::fib_sequential(n));
            bt_finish(S);
            return;
        }
        if (threadIdx.x == 0) {
            *reinterpret_cast<int4*>(bt_spawn(A, S, K_FIB, nullptr, nullptr, false, false)) = make_int4(n - 1, 0, 0, 4);
            *reinterpret_cast<int4*>(bt_spawn(A, S, K_FIB, nullptr, nullptr, false, false)) = make_int4(n - 2, 0, 0, 8);
        }
        if (bt_join(A, S, 1)) return;
        st = 1;
    }
    if (st == 1) {
        if (threadIdx.x == 0) bt_return_i32(A, S, fr.w & prog::kFibSlotMask, fr.y + fr.z);
    } else if (threadIdx.x == 0) {
        GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.task, -1, st, 1);
    }
    bt_finish(S);
}

// gtap_nq.cu:10-55 (no taskwait): one block per row task, thread 0 forks.
__device__ void nq_task(const Arena& A, BlockShared& S) {
    const int4 fr = S.w0;
    const int row = fr.x & 0xFF, n = (fr.x >> 8) & 0xFF, cutoff = (fr.x >> 16) & 0xFF;
    const unsigned column = (unsigned)fr.y, left = (unsigned)fr.z, right = (unsigned)fr.w;
    if (threadIdx.x == 0) {
        if (row > cutoff) {
            bt_add_value(S, prog::nq_serial(row, column, left, right, n));
        } else {
            const unsigned mask = (n < 32 ? (1u << n) - 1u : 0xFFFFFFFFu);
            unsigned avail = mask & ~(column | left | right);
            while (avail) {
                const unsigned p = avail & (0u - avail);
                avail -= p;
                *reinterpret_cast<int4*>(bt_spawn(A, S, K_NQ, nullptr, nullptr, false, true)) =
                    make_int4(fr.x + 1, (int)(column | p), (int)((left | p) << 1), (int)((right | p) >> 1));
            }
        }
    }
    bt_finish(S);
}

// asynchronous_bfs_block.cu:19-31: the block strides over v's adjacency (or
// the edge range [start, end) of a split task), relaxes every neighbour and
// spawns a task for each one it improved.
__device__ void bfs_task(const Arena& A, BlockShared& S) {
    const gtap_root& rd = bt_root(A, S);
    const int* row = reinterpret_cast<const int*>(rd.p0);
    const int* col = reinterpret_cast<const int*>(rd.p1);
    int* depth = reinterpret_cast<int*>(rd.p2);
    const int v = S.w0.x;
    int start = S.w0.y, end = S.w0.z;
    if (start < 0) {
        start = __ldg(row + v);
        end = __ldg(row + v + 1);
    }
    const int nd = ld_cg(depth + v) + 1;
    for (int e = start + (int)threadIdx.x; e < end; e += blockDim.x) {
        const int u = __ldg(col + e);
        if (atomicMin(depth + u, nd) > nd)
            *reinterpret_cast<int4*>(bt_spawn(A, S, K_BFS, nullptr, nullptr, false, true)) = make_int4(u, -1, -1, 0);
    }
    bt_finish(S);
}

// tree sum (binary_tree_thread.cu:63-114 shape, int64): subtrees of at most
// the cutoff are walked by thread 0, larger ones fork both children and join.
__device__ void treesum_task(const Arena& A, BlockShared& S) {
    const gtap_root& rd = bt_root(A, S);
    const int* left = reinterpret_cast<const int*>(rd.p0);
    const int* right = reinterpret_cast<const int*>(rd.p1);
    const int* value = reinterpret_cast<const int*>(rd.p2);
    const int* size = reinterpret_cast<const int*>(rd.p3);
    const int4 w0 = S.w0, w1 = S.w1;
    const int node = w0.x, slot = w0.y;
    int st = bt_state(S);
    long long a = 0, b = 0;
    if (st == 0) {
        const int sz = __ldg(size + node);
        if (sz <= rd.i1) {
            if (threadIdx.x == 0) {
                bool bad = false;
                bt_return_i64(A, S, slot, prog::tree_serial(left, right, value, size, node, sz, &bad));
                if (bad) GTAP_ERROR(A, ERR_INVALID_ARGUMENT, S.task, -1, node, sz);
            }
            bt_finish(S);
            return;
        }
        if (threadIdx.x == 0) {
            prog::TreeFrame* f = reinterpret_cast<prog::TreeFrame*>(frame_of(A, S.task));
            f->a = 0;
            f->b = 0;
            const int l = __ldg(left + node), r = __ldg(right + node);
            if (l >= 0) *reinterpret_cast<int4*>(bt_spawn(A, S, K_TREESUM, nullptr, nullptr, false, false)) = make_int4(l, 8, 0, 0);
            if (r >= 0) *reinterpret_cast<int4*>(bt_spawn(A, S, K_TREESUM, nullptr, nullptr, false, false)) = make_int4(r, 16, 0, 0);
        }
        if (bt_join(A, S, 1)) return;
        st = 1;   // no child: both sums are zero
    } else {
        a = (long long)(((unsigned long long)(unsigned)w0.w << 32) | (unsigned)w0.z);
        b = (long long)(((unsigned long long)(unsigned)w1.y << 32) | (unsigned)w1.x);
    }
    if (st == 1) {
        if (threadIdx.x == 0) bt_return_i64(A, S, slot, (long long)__ldg(value + node) + a + b);
    } else if (threadIdx.x == 0) {
        GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.task, -1, st, 1);
    }
    bt_finish(S);
}

}  // namespace bprog

// The built-in program of the block kernel: the thread-mode root table, with
// leaf sizes bounded by what one block stages in shared memory.
struct BlockProgram {
    static constexpr int kSmemInts = bprog::kSmemInts;
    static constexpr bool kFuncTable = false;
    __device__ static int root_kind(int k) { return BuiltinProgram::root_kind(k); }
    __device__ static bool root_args_ok(const gtap_root& rd) {
        if (!BuiltinProgram::root_args_ok(rd)) return false;
        switch (rd.kind) {
            // leaves hold n < sort cutoff keys and merges alen + blen < merge cutoff
            case GTAP_KIND_CILKSORT: return rd.i0 <= bprog::kLeafMax + 1 && rd.i1 <= bprog::kLeafMax + 1;
            // leaves hold n <= cutoff keys
            case GTAP_KIND_MERGESORT: return rd.i0 <= bprog::kLeafMax && rd.i1 <= bprog::kLeafMax + 1;
            default: return true;
        }
    }
    __device__ static void init_root(const Arena& A, const gtap_root& rd, void* frame) {
        BuiltinProgram::init_root(A, rd, frame);
    }
    __device__ static void exec(const Arena& A, BlockShared& S, int tid, int* smem) {
        switch (S.kind) {
            case prog::K_FIB: bprog::fib_task(A, S); break;
            case prog::K_NQ: bprog::nq_task(A, S); break;
            case prog::K_CILKSORT: bprog::cilksort_task(A, S, smem); break;
            case prog::K_CILKMERGE: bprog::cilkmerge_task(A, S, smem); break;
            case prog::K_MERGESORT: bprog::mergesort_task(A, S, smem); break;
            case prog::K_BFS: bprog::bfs_task(A, S); break;
            case prog::K_TREESUM: bprog::treesum_task(A, S); break;
            default:
                if (threadIdx.x == 0) GTAP_ERROR(A, ERR_INVALID_KIND, tid, -1, S.kind, 0);
                bt_finish(S);
                break;
        }
    }
};

// 2048 threads per SM at any block size up to kBMaxThreads: at most 32
// registers a thread, so eight 256-thread workers fit on every SM.
template <class Prog>
__global__ void __launch_bounds__(kBMaxThreads, 2048 / kBMaxThreads) block_worker_kernel(const __grid_constant__ Arena A) {
    __shared__ BlockShared S;
    extern __shared__ __align__(16) int block_smem[];
    block_worker<Prog>(A, S, block_smem);
}

}  // namespace gtap
