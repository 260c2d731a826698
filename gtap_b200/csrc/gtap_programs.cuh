// gtap_programs.cuh -- the built-in task functions, hand-lowered into the
// switch-statement state machine that clang-gtap emits for
// `#pragma gtap task` / `taskwait` / `queue(expr)` (the compiler itself is an
// empty submodule in the reference, so the lowering is written out here).
//
// Each task follows the reference's task body (paths relative to the
// reference project root); the cited lines are the algorithm being lowered.
// Two lowering choices differ from the reference's generated code but not its
// results:
//   * a child writes its return value straight into the parent's frame (the
//     byte offset travels in the child frame) instead of the parent reading a
//     retained child frame after the join;
//   * tasks that never taskwait (n-queens, BFS) spawn "detached" children,
//     which is what GTAP_ASSUME_NO_TASKWAIT builds do in the reference.
#pragma once
#include "gtap_thread_sched.cuh"

namespace gtap {
namespace prog {

enum : int { K_FIB = 1, K_NQ = 2, K_CILKSORT = 3, K_CILKMERGE = 4, K_MERGESORT = 5, K_BFS = 6, K_TREESUM = 7 };

constexpr int kFrameBytes = 32;

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ const gtap_root& root_of(const Arena& A, const WarpShared& S) {
    return A.roots[S.l_root[lane_id()]];
}

// Return an int value: into the parent's frame at byte offset `slot`, or into
// the root result for a root task.
__device__ __forceinline__ void return_i32(const Arena& A, const WarpShared& S, int slot, int value) {
    const int parent = S.l_parent[lane_id()];
    if (parent >= 0) {
        *reinterpret_cast<int*>(reinterpret_cast<char*>(frame_of(A, parent)) + slot) = value;
    } else {
        A.results[S.l_root[lane_id()]].value = value;
    }
}
__device__ __forceinline__ void return_i64(const Arena& A, const WarpShared& S, int slot, long long value) {
    const int parent = S.l_parent[lane_id()];
    if (parent >= 0) {
        *reinterpret_cast<long long*>(reinterpret_cast<char*>(frame_of(A, parent)) + slot) = value;
    } else {
        A.results[S.l_root[lane_id()]].value = value;
    }
}

// ---------------------------------------------------------------------------
// fib -- evaluation/2-comparison/fib/gtap_fib.cu:10-22 (cutoff 0) and
// evaluation/3-epaq/fib/fib_queue_1.cu:9-26 (n < cutoff runs fib_sequential);
// EPAQ variant fib_queue_3.cu:16-26 when root.i2 != 0 and Q >= 3.
// ---------------------------------------------------------------------------
struct FibFrame {
    int n;
    int a;     // result of fib(n-1), written by child 1
    int b;     // result of fib(n-2), written by child 2
    int slot;  // bits 0-7: byte offset of this task's result in its parent's frame; the root's settings,
               // copied to every task so none reads the root descriptor: bits 8-15 the serial cutoff
               // (clamped to 0..65, n <= 64), bit 16 the EPAQ variant (root.i2 != 0 and 3+ queues)
};
constexpr int kFibSlotMask = 0xFF;

// fib_queue_1.cu:9-14: visits the same call tree as the reference's doubly
// recursive fib_sequential (every node n >= 2 expands into n-1 and n-2, every
// leaf adds n), but as a loop: no device stack, so no depth limit from the
// per-thread stack size.  The walk goes to n-2 first and leaves n-1 pending;
// pending values along the current path strictly decrease towards the top of
// the stack, so the stack is a bit set and its top is the lowest set bit.
// Valid for n <= 64 (roots are checked); the sum wraps like the reference's int.
static __device__ __noinline__ int fib_sequential(int n) {
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

// kPair: both children through rt_spawn_pair (one id-cache and one staging
// claim for the two); used in the fib / n-queens kernel, whose registers have
// room for it (the other kernels spill with it).
template <bool kPair>
__device__ __forceinline__ void fib_task(const Arena& A, WarpShared& S, void* frame, const int4& w0) {
    FibFrame* f = reinterpret_cast<FibFrame*>(frame);
    int4 fr = w0;   // {n, a, b, slot}, loaded with the header
    switch (rt_state(S)) {
        case 0: {
            const int n = fr.x, cutoff = (fr.w >> 8) & 0xFF;
            if (n < 2) {
                return_i32(A, S, fr.w & kFibSlotMask, n);
                rt_finish(S);
                return;
            }
            if (n < cutoff) {
                return_i32(A, S, fr.w & kFibSlotMask, fib_sequential(n));
                rt_finish(S);
                return;
            }
            const bool epaq = (fr.w >> 16) & 1;
            int cc = 0;
            void* c1;
            void* c2;
            if (kPair && !epaq) {
                rt_spawn_pair(A, S, K_FIB, &cc, &c1, &c2);
            } else {
                c1 = rt_spawn(A, S, K_FIB, epaq ? ((n - 1) < cutoff ? 1 : 0) : 0, &cc, nullptr, false, false);
                c2 = rt_spawn(A, S, K_FIB, epaq ? ((n - 2) < cutoff ? 1 : 0) : 0, &cc, nullptr, false, false);
            }
            const int settings = fr.w & ~kFibSlotMask;
            *reinterpret_cast<int4*>(c1) = make_int4(n - 1, 0, 0, settings | 4);
            *reinterpret_cast<int4*>(c2) = make_int4(n - 2, 0, 0, settings | 8);
            // the continuation below (return a + b) is the kJoinSumBit one: the
            // child that completes the join may run it in place of resuming
            // this task (gtap_config::join_walk)
            if (rt_join(A, S, cc, 1, epaq ? 2 : 0, true)) return;
            fr = ld_data_v4(f);
        }
        // fallthrough
        case 1: {
            return_i32(A, S, fr.w & kFibSlotMask, fr.y + fr.z);
            rt_finish(S);
            return;
        }
        default:
            GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.l_tid[lane_id()], -1, rt_state(S), 1);
            rt_finish(S);
            return;
    }
}

// ---------------------------------------------------------------------------
// n-queens -- evaluation/2-comparison/nq/gtap_nq.cu:10-55 (no-taskwait build)
// ---------------------------------------------------------------------------
struct NqFrame {
    int meta;          // row | n << 8 | cutoff_depth << 16
    unsigned column;
    unsigned left;
    unsigned right;
};

// gtap_nq.cu:10-23 serial_search, returning the count instead of atomics.
// The same depth-first search over rows row..n-1, written as a loop so it
// needs no device stack.  The diagonal masks are kept in 64-bit registers
// (left unshifted, right shifted up by 32) so that placing a queen can be
// undone exactly: no bit falls off either end within 32 rows.  Only the
// column chosen on each row is stored; the candidates still to try on a row
// are the free columns above that choice (the search takes the lowest first).
// The last row counts its free columns instead of visiting each one.
// Valid for 0 <= row <= n <= 32 (roots are checked).
static __device__ __noinline__ int nq_serial(int row, unsigned column, unsigned left, unsigned right, int n) {
    if (row >= n) return row == n ? 1 : 0;
    const unsigned mask = (n < 32 ? (1u << n) - 1u : 0xFFFFFFFFu);
    unsigned long long L = left, R = (unsigned long long)right << 32;
    unsigned C = column;
    unsigned char chosen[32];
    const int last = n - row - 1;   // depth of the last row below `row`
    int d = 0;
    int total = 0;
    unsigned avail = mask & ~(C | (unsigned)L | (unsigned)(R >> 32));
    for (;;) {
        if (d == last) {
            total += __popc(avail);
            avail = 0;
        }
        if (avail) {
            const unsigned p = avail & (0u - avail);
            chosen[d] = (unsigned char)(__ffs((int)p) - 1);
            C |= p;
            L = (L | p) << 1;
            R = (R | ((unsigned long long)p << 32)) >> 1;
            ++d;
            avail = mask & ~(C | (unsigned)L | (unsigned)(R >> 32));
            continue;
        }
        if (d == 0) break;
        --d;
        const unsigned p = 1u << chosen[d];
        C &= ~p;
        L = (L >> 1) & ~(unsigned long long)p;
        R = (R << 1) & ~((unsigned long long)p << 32);
        avail = mask & ~(C | (unsigned)L | (unsigned)(R >> 32)) & ~((p << 1) - 1u);
    }
    return total;
}

__device__ __forceinline__ void nq_task(const Arena& A, WarpShared& S, void* frame, const int4& w0) {
    (void)frame;
    const int4 fr = w0;
    const int row = fr.x & 0xFF, n = (fr.x >> 8) & 0xFF, cutoff = (fr.x >> 16) & 0xFF;
    const unsigned column = (unsigned)fr.y, left = (unsigned)fr.z, right = (unsigned)fr.w;
    if (row > cutoff) {
        S.l_value[lane_id()] += nq_serial(row, column, left, right, n);
        rt_finish(S);
        return;
    }
    const unsigned mask = (n < 32 ? (1u << n) - 1u : 0xFFFFFFFFu);
    unsigned avail = mask & ~(column | left | right);
    while (avail) {
        unsigned p = avail & (0u - avail);
        avail -= p;
        NqFrame* c = reinterpret_cast<NqFrame*>(rt_spawn(A, S, K_NQ, 0, nullptr, nullptr, false, true));
        *reinterpret_cast<int4*>(c) =
            make_int4(fr.x + 1, (int)(column | p), (int)((left | p) << 1), (int)((right | p) >> 1));
    }
    rt_finish(S);
}

// ---------------------------------------------------------------------------
// cilksort / cilkmerge -- examples/cilksort/cilksort.cu:17-164
// ---------------------------------------------------------------------------
struct SortFrame {
    int* arr;          // sorted in place (cilksort.cu `arr`)
    int* tmp;          // scratch (cilksort.cu `tmp`)
    const int* src;    // unsorted input read by the leaves (so repeated runs need no restore)
    int n;
    int pad;
};
struct MergeFrame {
    const int* a;
    const int* b;
    int* dst;
    int alen;
    int blen;
};
static_assert(sizeof(SortFrame) <= kFrameBytes && sizeof(MergeFrame) <= kFrameBytes, "frame size");

// ---------------------------------------------------------------------------
// Warp-cooperative leaves.  A leaf sort (cilksort.cu:51-86 sort_small_device,
// mergesort.cu:15-32 mergesort_rec_device) or leaf merge (cilksort.cu:17-36
// seqmerge) does not run in the lane that reached it: the lane marks its task
// in its lane flags and returns, and after the round's task bodies the whole warp
// works through the marked tasks one at a time (warp_leaves below), before any
// parent is told that they finished.  Keys move as coalesced 128-byte rows,
// sorting uses shuffles instead of a per-thread register network, and a leaf
// may have any length.  The output is the same sorted sequence.
// ---------------------------------------------------------------------------
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ void mark_leaf(WarpShared& S) { S.l_flags[lane_id()] |= kLaneLeaf; }

// Bitonic sort of the 64 keys held two per lane (key i = r * 32 + lane in
// v[r]), ascending.
__device__ __forceinline__ void warp_bitonic64(int& v0, int& v1) {
    const unsigned lane = lane_id();
#pragma unroll
    for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j == 32) {   // k == 64: key lane pairs with key lane + 32, ascending
                const int lo = min(v0, v1), hi = max(v0, v1);
                v0 = lo;
                v1 = hi;
            } else {
                const int p0 = __shfl_xor_sync(kFull, v0, j);
                const int p1 = __shfl_xor_sync(kFull, v1, j);
                const bool lower = (lane & (unsigned)j) == 0;
                const bool up0 = (lane & (unsigned)k) == 0;
                const bool up1 = ((lane + 32u) & (unsigned)k) == 0;
                v0 = (lower == up0) ? min(v0, p0) : max(v0, p0);
                v1 = (lower == up1) ? min(v1, p1) : max(v1, p1);
            }
        }
    }
}

// dst[0, alen + blen) = merge of sorted a and b (a first among equal keys).
// Each lane produces 8 consecutive outputs per 256-output tile, starting at
// the merge-path split of its first output.
static __device__ __noinline__ void warp_merge(const int* a, int alen, const int* b, int blen, int* dst) {
    const int lane = (int)lane_id();
    const int total = alen + blen;
    for (int t0 = 0; t0 < total; t0 += 256) {
        const int d = t0 + lane * 8;
        if (d < total) {
            int lo = max(0, d - blen), hi = min(d, alen);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (ld_data(a + mid) <= ld_data(b + (d - 1 - mid))) lo = mid + 1;
                else hi = mid;
            }
            int i = lo, j = d - lo;
            const int m = min(8, total - d);
            int av = i < alen ? ld_data(a + i) : 0, bv = j < blen ? ld_data(b + j) : 0;
            for (int e = 0; e < m; ++e) {
                const bool take_a = j >= blen || (i < alen && av <= bv);
                if (take_a) {
                    dst[d + e] = av;
                    if (++i < alen) av = ld_data(a + i);
                } else {
                    dst[d + e] = bv;
                    if (++j < blen) bv = ld_data(b + j);
                }
            }
        }
    }
}

// Leaves of at most kLeafKeys keys go through the warp's shared-memory leaf
// buffers: gtap_config.leaf_batch input buffers of kLeafKeys keys and one
// output buffer.
// The keys of a batch of leaves are copied in with cp.async (every copy of
// every leaf of the batch in flight at once: one round trip per batch, no
// registers held), merge-path searches and merges read shared memory, and
// results leave with coalesced stores.  A merge leaf done in
// global memory costs a dependent round trip per binary-search step and per
// merged key, and leaves done one at a time a round trip each.  The loops
// stay rolled and the two leaf routines inline: unrolled loops measured
// slower even with the sort kernel alone on the SMs (the instruction cache
// again), and calls out of line slower than inlined code (the 2^10-2^20-key
// cilksort roots of the seed-42 mix: 26.7 ms out of line, 25.0 ms inline,
// 28.1 ms inline and unrolled).
constexpr int kLeafKeys = 256;

__device__ __forceinline__ void cp_async4(int* smem_dst, const int* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Starts copying buf[0, total) = a[0, alen) ++ b[0, total - alen); the
// caller waits (cp_async_wait_all + __syncwarp) before reading buf.
__device__ __forceinline__ void leaf_issue(const int* a, int alen, const int* b, int total, int* buf) {
#pragma unroll 1
    for (int i = (int)lane_id(); i < total; i += 32) cp_async4(buf + i, i < alen ? a + i : b + (i - alen));
}

// out[d, d + 8) (clipped to alen + blen) = outputs d.. of the merge of
// sorted a[0, alen) and b[0, blen) (merge path; a's key first among equal keys).
__device__ __forceinline__ void merge_path8(const int* a, int alen, const int* b, int blen, int d, int* out) {
    int lo = max(0, d - blen), hi = min(d, alen);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= b[d - 1 - mid]) lo = mid + 1;
        else hi = mid;
    }
    int i = lo, j = d - lo;
    const int end = min(d + 8, alen + blen);
#pragma unroll 1
    for (int e = d; e < end; ++e) {
        const bool take_a = j >= blen || (i < alen && a[i] <= b[j]);
        out[e] = take_a ? a[i++] : b[j++];
    }
}

__device__ __forceinline__ void leaf_store(const int* buf, int total, int* dst) {
#pragma unroll 1
    for (int i = (int)lane_id(); i < total; i += 32) dst[i] = buf[i];
}

// in = a[0, alen) ++ b[0, blen), both sorted: dst[0, alen + blen) = their
// merge (the sequence warp_merge writes), through out.
__device__ __forceinline__ void leaf_merge_out(const int* in, int alen, int blen, int* out, int* dst) {
    __syncwarp();   // out's previous contents were stored already
    const int d0 = (int)lane_id() * 8;
    if (d0 < alen + blen) merge_path8(in, alen, in + alen, blen, d0, out);
    __syncwarp();
    leaf_store(out, alen + blen, dst);
}

// dst[0, n) = in[0, n) sorted: 64-key runs sorted in place by
// warp_bitonic64, then merge passes of doubling width between in and out.
__device__ __forceinline__ void leaf_sort_out(int* in, int n, int* out, int* dst) {
    const int lane = (int)lane_id();
    __syncwarp();   // out's previous contents were stored already
#pragma unroll 1
    for (int c = 0; c < n; c += 64) {
        int v0 = c + lane < n ? in[c + lane] : 0x7fffffff;
        int v1 = c + lane + 32 < n ? in[c + lane + 32] : 0x7fffffff;
        warp_bitonic64(v0, v1);   // keys past n sort last and are never stored
        if (c + lane < n) in[c + lane] = v0;
        if (c + lane + 32 < n) in[c + lane + 32] = v1;
    }
    __syncwarp();
    int* from = in;
    int* to = out;
#pragma unroll 1
    for (int w = 64; w < n; w <<= 1) {
        const int d0 = lane * 8;
        if (d0 < n) {
            const int s = d0 / (2 * w) * (2 * w);
            const int alen = min(w, n - s), blen = min(w, n - s - alen);
            merge_path8(from + s, alen, from + s + alen, blen, d0 - s, to + s);
        }
        __syncwarp();
        int* t = from;
        from = to;
        to = t;
    }
    leaf_store(from, n, dst);
}

// out[0, n) = in[0, n) sorted; scr is n keys of scratch (in may alias out).
// 64-key runs by warp_bitonic64, then merge passes of doubling width that
// alternate between scr and out so the last one lands in out.
static __device__ __noinline__ void warp_sort(const int* in, int* out, int* scr, int n) {
    const int lane = (int)lane_id();
    const int runs = (n + 63) >> 6;
    int passes = 0;
    for (int w = 1; w < runs; w <<= 1) ++passes;
    int* from = (passes & 1) ? scr : out;
    int* to = (passes & 1) ? out : scr;
    for (int c = 0; c < n; c += 64) {
        const int m = min(64, n - c);
        int v0 = lane < m ? ld_data(in + c + lane) : 0x7fffffff;
        int v1 = lane + 32 < m ? ld_data(in + c + lane + 32) : 0x7fffffff;
        __syncwarp();   // every key of this run is read before any is written (in may alias out)
        warp_bitonic64(v0, v1);
        if (lane < m) from[c + lane] = v0;
        if (lane + 32 < m) from[c + lane + 32] = v1;
    }
    for (int width = 64; width < n; width <<= 1) {
        __syncwarp();
        for (int s = 0; s < n; s += 2 * width) {
            const int alen = min(width, n - s);
            const int blen = min(width, n - s - alen);
            warp_merge(from + s, alen, from + s + alen, blen, to + s);
        }
        int* t = from;
        from = to;
        to = t;
    }
    __syncwarp();
}

// cilksort.cu:38-49: largest index with x[idx] <= val.  The answer is the
// binary search's.  quad: three probes per step, loaded together, keep a
// quarter of the interval, so a split costs half the dependent loads (10 steps
// instead of 20 for 2^20 keys) for 1.5x the loads and more instructions.
// Invariant: x[low] <= val (or low == -1) and x[high] > val (or high == len).
__device__ __forceinline__ int bsearch_le(const int* x, int len, int val, bool quad) {
    int low = -1, high = len;
    while (quad && high - low > 4) {
        const int q = (high - low) / 4;
        const int m1 = low + q, m2 = low + 2 * q, m3 = low + 3 * q;   // low < m1 < m2 < m3 < high
        const int v1 = ld_data(x + m1), v2 = ld_data(x + m2), v3 = ld_data(x + m3);
        if (v3 <= val) {
            low = m3;
        } else if (v2 <= val) {
            low = m2;
            high = m3;
        } else if (v1 <= val) {
            low = m1;
            high = m2;
        } else {
            high = m1;
        }
    }
    while (low + 1 < high) {
        int mid = (low + high) / 2;
        if (ld_data(x + mid) <= val) low = mid;
        else high = mid;
    }
    return low;
}

__device__ __forceinline__ void spawn_merge(const Arena& A, WarpShared& S, int* cc, const int* a, int alen,
                                            const int* b, int blen, int* dst) {
    MergeFrame* m = reinterpret_cast<MergeFrame*>(rt_spawn(A, S, K_CILKMERGE, 0, cc, nullptr, false, false));
    m->a = a;
    m->b = b;
    m->dst = dst;
    m->alen = alen;
    m->blen = blen;
}

// cilksort.cu:89-125
__device__ __forceinline__ void cilkmerge_task(const Arena& A, WarpShared& S, void* frame, const int4& w0,
                                               const int4& w1) {
    if (rt_state(S) != 0) {  // resumed after the taskwait: nothing left to do
        rt_finish(S);
        return;
    }
    const MergeFrame* f = reinterpret_cast<const MergeFrame*>(frame);
    const int* a = reinterpret_cast<const int*>((unsigned long long)(unsigned)w0.x | ((unsigned long long)(unsigned)w0.y << 32));
    const int* b = reinterpret_cast<const int*>((unsigned long long)(unsigned)w0.z | ((unsigned long long)(unsigned)w0.w << 32));
    int* dst = reinterpret_cast<int*>((unsigned long long)(unsigned)w1.x | ((unsigned long long)(unsigned)w1.y << 32));
    int alen = w1.z, blen = w1.w;
    (void)f;
    if (alen < blen) {
        const int* t = a; a = b; b = t;
        int tl = alen; alen = blen; blen = tl;
    }
    const gtap_root& rd = root_of(A, S);
    const int cutoff = rd.i1;
    if (blen == 0 || alen + blen < cutoff) {   // a copy or a leaf merge: warp_leaves does it
        mark_leaf(S);
        rt_finish(S);
        return;
    }
    const int as = (alen + 1) / 2;
    // Sorts of 2^22 keys or more search their splits four ways: their depth of
    // dependent splits sets their time (mergesort of 2^24 keys 6.27 -> 5.85 ms,
    // cilksort of 10^7..10^8 keys 2-5 % faster).  Smaller sorts, such as the
    // mix's (at most 2^20 keys), run many short searches at once, where the
    // extra loads and instructions cost more (its sort launch 22.5 -> 22.8 ms).
    const int bs = bsearch_le(b, blen, ld_data(a + as - 1), rd.n >= (1ll << 22)) + 1;
    int cc = 0;
    spawn_merge(A, S, &cc, a, as, b, bs, dst);
    spawn_merge(A, S, &cc, a + as, alen - as, b + bs, blen - bs, dst + as + bs);
    if (rt_join(A, S, cc, 1, 0)) return;
    rt_finish(S);
}

__device__ __forceinline__ void spawn_sort(const Arena& A, WarpShared& S, int* cc, int* arr, int* tmp,
                                           const int* src, int n) {
    SortFrame* c = reinterpret_cast<SortFrame*>(rt_spawn(A, S, K_CILKSORT, 0, cc, nullptr, false, false));
    c->arr = arr;
    c->tmp = tmp;
    c->src = src;
    c->n = n;
}

// cilksort.cu:127-164
__device__ __forceinline__ void cilksort_task(const Arena& A, WarpShared& S, void* frame, const int4& w0,
                                              const int4& w1) {
    (void)frame;
    int* arr = reinterpret_cast<int*>((unsigned long long)(unsigned)w0.x | ((unsigned long long)(unsigned)w0.y << 32));
    int* tmp = reinterpret_cast<int*>((unsigned long long)(unsigned)w0.z | ((unsigned long long)(unsigned)w0.w << 32));
    const int* src = reinterpret_cast<const int*>((unsigned long long)(unsigned)w1.x | ((unsigned long long)(unsigned)w1.y << 32));
    const int n = w1.z;
    const int len12 = n / 2, len1 = len12 / 2, len2 = len12 - len1;
    const int len34 = n - len12, len3 = len34 / 2, len4 = len34 - len3;
    int cc = 0;
    switch (rt_state(S)) {
        case 0: {
            const int sort_cutoff = root_of(A, S).i0;
            if (n < sort_cutoff) {   // leaf: warp_leaves sorts src into arr, tmp as scratch
                if (n > 0) mark_leaf(S);
                rt_finish(S);
                return;
            }
            spawn_sort(A, S, &cc, arr, tmp, src, len1);
            spawn_sort(A, S, &cc, arr + len1, tmp + len1, src + len1, len2);
            spawn_sort(A, S, &cc, arr + len12, tmp + len12, src + len12, len3);
            spawn_sort(A, S, &cc, arr + len12 + len3, tmp + len12 + len3, src + len12 + len3, len4);
            if (rt_join(A, S, cc, 1, 0)) return;
        }
        // fallthrough
        case 1: {
            cc = 0;
            spawn_merge(A, S, &cc, arr, len1, arr + len1, len2, tmp);
            spawn_merge(A, S, &cc, arr + len12, len3, arr + len12 + len3, len4, tmp + len12);
            if (rt_join(A, S, cc, 2, 0)) return;
        }
        // fallthrough
        case 2: {
            cc = 0;
            spawn_merge(A, S, &cc, tmp, len12, tmp + len12, len34, arr);
            if (rt_join(A, S, cc, 3, 0)) return;
        }
        // fallthrough
        case 3:
            rt_finish(S);
            return;
        default:
            GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.l_tid[lane_id()], -1, rt_state(S), 3);
            rt_finish(S);
            return;
    }
}

// ---------------------------------------------------------------------------
// mergesort -- examples/mergesort/mergesort.cu:34-50 recursion (n > cutoff
// forks the two halves [left, mid] / [mid+1, right]); the merge after the
// taskwait is the parallel cilkmerge above, with ping-pong buffers instead of
// merge_device's single-thread merge and copy-back.
// ---------------------------------------------------------------------------
struct MsFrame {
    const int* in;   // unsorted input
    int* out;        // sorted output
    int* tmp;        // scratch of the same size
    int n;
    int pad;
};
static_assert(sizeof(MsFrame) <= kFrameBytes, "frame size");

__device__ __forceinline__ void mergesort_task(const Arena& A, WarpShared& S, void* frame, const int4& w0,
                                               const int4& w1) {
    (void)frame;
    const int* in = reinterpret_cast<const int*>((unsigned long long)(unsigned)w0.x | ((unsigned long long)(unsigned)w0.y << 32));
    int* out = reinterpret_cast<int*>((unsigned long long)(unsigned)w0.z | ((unsigned long long)(unsigned)w0.w << 32));
    int* tmp = reinterpret_cast<int*>((unsigned long long)(unsigned)w1.x | ((unsigned long long)(unsigned)w1.y << 32));
    const int n = w1.z;
    const int nl = (n + 1) / 2;   // [left, mid] holds ceil(n/2) keys
    int cc = 0;
    switch (rt_state(S)) {
        case 0: {
            const int cutoff = root_of(A, S).i0;
            if (n <= cutoff || n <= 1) {   // leaf: warp_leaves sorts in into out, tmp as scratch
                if (n > 0) mark_leaf(S);
                rt_finish(S);
                return;
            }
            // children sort into tmp, using out as their scratch
            MsFrame* c1 = reinterpret_cast<MsFrame*>(rt_spawn(A, S, K_MERGESORT, 0, &cc, nullptr, false, false));
            c1->in = in;
            c1->out = tmp;
            c1->tmp = out;
            c1->n = nl;
            MsFrame* c2 = reinterpret_cast<MsFrame*>(rt_spawn(A, S, K_MERGESORT, 0, &cc, nullptr, false, false));
            c2->in = in + nl;
            c2->out = tmp + nl;
            c2->tmp = out + nl;
            c2->n = n - nl;
            if (rt_join(A, S, cc, 1, 0)) return;
        }
        // fallthrough
        case 1: {
            cc = 0;
            spawn_merge(A, S, &cc, tmp, nl, tmp + nl, n - nl, out);
            if (rt_join(A, S, cc, 2, 0)) return;
        }
        // fallthrough
        case 2:
            rt_finish(S);
            return;
        default:
            GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.l_tid[lane_id()], -1, rt_state(S), 2);
            rt_finish(S);
            return;
    }
}

// ---------------------------------------------------------------------------
// asynchronous BFS -- examples/asynchronous_bfs/asynchronous_bfs_thread.cu:19-49
// (atomicMin relaxation, spawn per improved vertex).  A vertex whose edge
// range exceeds the split threshold is halved recursively, so a task never
// spawns more than max(2, threshold) children.
// ---------------------------------------------------------------------------
struct BfsFrame {
    int v;
    int start;   // -1: whole adjacency of v
    int end;
    int pad;
};

__device__ __forceinline__ void bfs_task(const Arena& A, WarpShared& S, void* frame, const int4& w0) {
    (void)frame;
    const int4 fr = w0;
    const gtap_root& rd = root_of(A, S);
    const int* row = reinterpret_cast<const int*>(rd.p0);
    const int* col = reinterpret_cast<const int*>(rd.p1);
    int* depth = reinterpret_cast<int*>(rd.p2);
    const int split = rd.i1 > 0 ? rd.i1 : 32;
    const int v = fr.x;
    int start = fr.y, end = fr.z;
    if (start < 0) {
        start = __ldg(row + v);
        end = __ldg(row + v + 1);
    }
    if (end - start > split) {
        const int mid = start + (end - start) / 2;
        BfsFrame* c1 = reinterpret_cast<BfsFrame*>(rt_spawn(A, S, K_BFS, 0, nullptr, nullptr, false, true));
        *reinterpret_cast<int4*>(c1) = make_int4(v, start, mid, 0);
        BfsFrame* c2 = reinterpret_cast<BfsFrame*>(rt_spawn(A, S, K_BFS, 0, nullptr, nullptr, false, true));
        *reinterpret_cast<int4*>(c2) = make_int4(v, mid, end, 0);
        rt_finish(S);
        return;
    }
    const int dv = ld_cg(depth + v);
    for (int e = start; e < end; ++e) {
        const int u = __ldg(col + e);
        const int nd = dv + 1;
        const int old = atomicMin(depth + u, nd);
        if (old > nd) {
            BfsFrame* c = reinterpret_cast<BfsFrame*>(rt_spawn(A, S, K_BFS, 0, nullptr, nullptr, false, true));
            *reinterpret_cast<int4*>(c) = make_int4(u, -1, -1, 0);
        }
    }
    rt_finish(S);
}

// ---------------------------------------------------------------------------
// tree sum over a pointer-linked binary tree (new served workload; the shape
// follows the reference's tree programs, examples/binary_tree/binary_tree_thread.cu:63-114,
// with int32 payloads summed into int64).
// ---------------------------------------------------------------------------
struct TreeFrame {
    int node;
    int slot;         // byte offset of this task's sum in its parent's frame
    long long a;      // left subtree sum
    long long b;      // right subtree sum
};
static_assert(sizeof(TreeFrame) <= kFrameBytes, "frame size");

// Sum of the subtree at `node`, whose size is `sz`, without recursion.  A
// subtree of at most 64 nodes is at most 64 deep, so a plain depth-first walk
// keeps at most 63 right children pending.  A larger subtree (a cutoff above
// 64) is walked into its smaller child first with the larger one pending, so
// each pending entry at least halves the subtree still being walked and at
// most 31 are pending.  A size array that contradicts the links can still fill
// the stack, and links with a cycle would walk forever; both set *bad (the
// walk stops after sz visits) and the sum is wrong, never a fault or a hang.
static __device__ __noinline__ long long tree_serial(const int* left, const int* right, const int* value,
                                                     const int* size, int node, int sz, bool* bad) {
    long long total = 0;
    int budget = sz;
    if (sz <= 64) {
        int stack[64];
        int sp = 0;
        stack[sp++] = node;
        while (sp > 0) {
            if (--budget < 0) { *bad = true; break; }
            const int v = stack[--sp];
            total += __ldg(value + v);
            const int l = __ldg(left + v), r = __ldg(right + v);
            if (r >= 0) {
                if (sp < 64) stack[sp++] = r;
                else *bad = true;
            }
            if (l >= 0) {
                if (sp < 64) stack[sp++] = l;
                else *bad = true;
            }
        }
        return total;
    }
    int pend_node[32], pend_size[32];
    int sp = 0;
    int v = node;
    for (;;) {
        if (--budget < 0) { *bad = true; break; }
        total += __ldg(value + v);
        const int l = __ldg(left + v), r = __ldg(right + v);
        if (l >= 0 && r >= 0) {
            const int sl = __ldg(size + l), sr = sz - 1 - sl;
            const bool left_first = sl <= sr;
            if (sp < 32) {
                pend_node[sp] = left_first ? r : l;
                pend_size[sp] = left_first ? sr : sl;
                ++sp;
            } else {
                *bad = true;
            }
            v = left_first ? l : r;
            sz = left_first ? sl : sr;
        } else if (l >= 0 || r >= 0) {
            v = l >= 0 ? l : r;
            sz -= 1;
        } else {
            if (sp == 0) break;
            --sp;
            v = pend_node[sp];
            sz = pend_size[sp];
        }
    }
    return total;
}

__device__ __forceinline__ void treesum_task(const Arena& A, WarpShared& S, void* frame, const int4& pw0,
                                             const int4& pw1) {
    TreeFrame* f = reinterpret_cast<TreeFrame*>(frame);
    const gtap_root& rd = root_of(A, S);
    const int* left = reinterpret_cast<const int*>(rd.p0);
    const int* right = reinterpret_cast<const int*>(rd.p1);
    const int* value = reinterpret_cast<const int*>(rd.p2);
    const int* size = reinterpret_cast<const int*>(rd.p3);
    int4 w0 = pw0, w1 = pw1;
    const int node = w0.x, slot = w0.y;
    switch (rt_state(S)) {
        case 0: {
            const int sz = __ldg(size + node);
            if (sz <= rd.i1) {
                bool bad = false;
                return_i64(A, S, slot, tree_serial(left, right, value, size, node, sz, &bad));
                if (bad) GTAP_ERROR(A, ERR_INVALID_ARGUMENT, S.l_tid[lane_id()], -1, node, sz);
                rt_finish(S);
                return;
            }
            f->a = 0;
            f->b = 0;
            int cc = 0;
            const int l = __ldg(left + node), r = __ldg(right + node);
            if (l >= 0) {
                TreeFrame* c = reinterpret_cast<TreeFrame*>(rt_spawn(A, S, K_TREESUM, 0, &cc, nullptr, false, false));
                *reinterpret_cast<int4*>(c) = make_int4(l, 8, 0, 0);
            }
            if (r >= 0) {
                TreeFrame* c = reinterpret_cast<TreeFrame*>(rt_spawn(A, S, K_TREESUM, 0, &cc, nullptr, false, false));
                *reinterpret_cast<int4*>(c) = make_int4(r, 16, 0, 0);
            }
            if (rt_join(A, S, cc, 1, 0)) return;
            w0 = ld_data_v4(frame);   // no child spawned: a, b are the zeros stored above
            w1 = ld_data_v4(reinterpret_cast<const char*>(frame) + 16);
        }
        // fallthrough
        case 1: {
            const long long a = (long long)(((unsigned long long)(unsigned)w0.w << 32) | (unsigned)w0.z);
            const long long b = (long long)(((unsigned long long)(unsigned)w1.y << 32) | (unsigned)w1.x);
            return_i64(A, S, slot, (long long)__ldg(value + node) + a + b);
            rt_finish(S);
            return;
        }
        default:
            GTAP_ERROR(A, ERR_INVALID_TASKWAIT, S.l_tid[lane_id()], -1, rt_state(S), 1);
            rt_finish(S);
            return;
    }
}

}  // namespace prog

// ---------------------------------------------------------------------------
// Program: dispatch by kind (a switch, not an indirect call)
// ---------------------------------------------------------------------------
// kSorts = false leaves the register-heavy sorting kinds out of the kernel,
// which lets fib / n-queens / BFS / tree launches run at higher occupancy;
// kGraphs = false also leaves out BFS and tree sums, so that a launch of fib
// and n-queens roots runs a kernel with two task bodies.  A task of a kind
// left out is recorded as ERR_INVALID_KIND.  (A sorting kernel without the
// fib, n-queens, BFS and tree bodies measured no faster on sort roots alone.)
template <bool kSorts, bool kGraphs = true>
struct BuiltinProgramT {
    static constexpr int kFrameBytes = prog::kFrameBytes;
    static constexpr bool kFrameWords = true;    // exec gets the first 32 frame bytes
    static constexpr bool kFuncTable = false;    // kinds are dispatched by the switch below
    static constexpr bool kJoinSum = true;       // fib's continuation runs at its join (kJoinSumBit)
    // extra passes on idle lanes (gtap_config::sub_rounds): only in the fib /
    // n-queens kernel, whose registers have room for the pass loop
    static constexpr bool kSubRounds = !kSorts && !kGraphs;
    static constexpr int kLeafKeys = kSorts ? prog::kLeafKeys : 0;   // keys per leaf buffer (0: no warp leaves)

    __device__ static int root_kind(int k) {
        switch (k) {
            case GTAP_KIND_FIB: return prog::K_FIB;
            case GTAP_KIND_NQ: return prog::K_NQ;
            case GTAP_KIND_CILKSORT: return prog::K_CILKSORT;
            case GTAP_KIND_MERGESORT: return prog::K_MERGESORT;
            case GTAP_KIND_BFS: return prog::K_BFS;
            case GTAP_KIND_TREESUM: return prog::K_TREESUM;
            default: return -1;
        }
    }

    // Argument ranges the built-in tasks rely on: fib's serial leaf handles
    // n <= 64, n-queens packs n and the cutoff into 8 bits with n <= 32
    // columns; the array kinds need their arrays, a count that fits int32 and
    // a start node inside it.  The recursions end only with a sort cutoff of
    // at least 2 (a one-key cilksort splits into 0, 0, 0 and 1 keys again) and
    // a merge cutoff of at least 3 (a merge of one key with one key splits
    // into itself).  A root that fails is recorded as an error and touches
    // none of its arrays.
    __device__ static bool root_args_ok(const gtap_root& rd) {
        switch (rd.kind) {
            case GTAP_KIND_FIB: return rd.i0 <= 64;
            case GTAP_KIND_NQ: return rd.i0 >= 0 && rd.i0 <= 32 && rd.i1 >= 0 && rd.i1 < 256;
            case GTAP_KIND_CILKSORT:
                if (rd.i0 < 2 || rd.i1 < 3) return false;
                return rd.n >= 0 && rd.n <= 0x7FFFFFFF && (rd.n == 0 || (rd.p0 && rd.p1 && rd.p2));
            case GTAP_KIND_MERGESORT:
                if (rd.i1 < 3) return false;
                return rd.n >= 0 && rd.n <= 0x7FFFFFFF && (rd.n == 0 || (rd.p0 && rd.p1 && rd.p2));
            case GTAP_KIND_BFS:
                return rd.p0 && rd.p1 && rd.p2 && rd.n > 0 && rd.n <= 0x7FFFFFFF && rd.i0 >= 0 && rd.i0 < rd.n;
            case GTAP_KIND_TREESUM:
                return rd.p0 && rd.p1 && rd.p2 && rd.p3 && rd.n > 0 && rd.n <= 0x7FFFFFFF && rd.i0 >= 0 &&
                       rd.i0 < rd.n;
            default: return true;
        }
    }

    __device__ static void init_root(const Arena& A, const gtap_root& rd, void* frame) {
        (void)A;
        int4* f = reinterpret_cast<int4*>(frame);
        switch (rd.kind) {
            case GTAP_KIND_FIB: {
                const int cutoff = rd.i1 < 0 ? 0 : (rd.i1 > 65 ? 65 : rd.i1);
                const int epaq = (rd.i2 != 0 && A.num_queues >= 3) ? 1 : 0;
                f[0] = make_int4(rd.i0, 0, 0, cutoff << 8 | epaq << 16);   // slot 0: the root's result
                break;
            }
            case GTAP_KIND_NQ:
                f[0] = make_int4(0 | (rd.i0 << 8) | (rd.i1 << 16), 0, 0, 0);
                break;
            case GTAP_KIND_CILKSORT: {
                prog::SortFrame* s = reinterpret_cast<prog::SortFrame*>(frame);
                s->arr = reinterpret_cast<int*>(rd.p1);
                s->tmp = reinterpret_cast<int*>(rd.p2);
                s->src = reinterpret_cast<const int*>(rd.p0);
                s->n = (int)rd.n;
                break;
            }
            case GTAP_KIND_MERGESORT: {
                prog::MsFrame* s = reinterpret_cast<prog::MsFrame*>(frame);
                s->in = reinterpret_cast<const int*>(rd.p0);
                s->out = reinterpret_cast<int*>(rd.p1);
                s->tmp = reinterpret_cast<int*>(rd.p2);
                s->n = (int)rd.n;
                break;
            }
            case GTAP_KIND_BFS: {
                // asynchronous_bfs_thread.cu:51-55: depth[source] = 0 before the entry task
                int* depth = reinterpret_cast<int*>(rd.p2);
                atomicExch(depth + rd.i0, 0);   // depth is otherwise only touched by atomics and L2 loads
                f[0] = make_int4(rd.i0, -1, -1, 0);
                break;
            }
            case GTAP_KIND_TREESUM:
                f[0] = make_int4(rd.i0, 0, 0, 0);
                f[1] = make_int4(0, 0, 0, 0);
                break;
            default:
                break;
        }
    }

    // Leaf work of the lanes in `mask`, done by the whole warp: each marked
    // lane's task kind and frame words (loaded with its header this round)
    // are broadcast, and the warp sorts or merges for that task.  Leaves of
    // at most kLeafKeys keys go in batches through the leaf buffers (S.lbuf:
    // A.leaf_buf input buffers and one output buffer), larger ones one at a
    // time through global memory.
    struct LeafArgs {
        int k, z1, q1;
        int *p0, *p1, *p2;
    };
    __device__ static LeafArgs leaf_args(int l, int kind, const int4& w0, const int4& w1) {
        LeafArgs a;
        a.k = __shfl_sync(prog::kFull, kind, l);
        const unsigned x0 = (unsigned)__shfl_sync(prog::kFull, w0.x, l), y0 = (unsigned)__shfl_sync(prog::kFull, w0.y, l);
        const unsigned z0 = (unsigned)__shfl_sync(prog::kFull, w0.z, l), q0 = (unsigned)__shfl_sync(prog::kFull, w0.w, l);
        const unsigned x1 = (unsigned)__shfl_sync(prog::kFull, w1.x, l), y1 = (unsigned)__shfl_sync(prog::kFull, w1.y, l);
        a.z1 = __shfl_sync(prog::kFull, w1.z, l);
        a.q1 = __shfl_sync(prog::kFull, w1.w, l);
        a.p0 = reinterpret_cast<int*>((unsigned long long)x0 | ((unsigned long long)y0 << 32));
        a.p1 = reinterpret_cast<int*>((unsigned long long)z0 | ((unsigned long long)q0 << 32));
        a.p2 = reinterpret_cast<int*>((unsigned long long)x1 | ((unsigned long long)y1 << 32));
        return a;
    }
    __device__ static void warp_leaves(const Arena& A, WarpShared& S, unsigned mask, int kind, const int4& w0,
                                       const int4& w1) {
        if constexpr (kSorts) {
            const unsigned lane = lane_id();
            int* buf = S.lbuf;
            const int nbuf = buf ? A.leaf_buf : 0;
            // frames: cilksort {arr, tmp, src, n}, cilkmerge {a, b, dst, alen, blen}, mergesort {in, out, tmp, n}
            bool small = false;
            if (nbuf > 0 && ((mask >> lane) & 1u))
                small = kind == prog::K_CILKMERGE ? w1.z + w1.w <= prog::kLeafKeys : w1.z <= prog::kLeafKeys;
            unsigned batch_of = __ballot_sync(prog::kFull, small);
            unsigned big = mask & ~batch_of;
            while (big) {
                const int l = __ffs(big) - 1;
                big &= big - 1;
                const LeafArgs a = leaf_args(l, kind, w0, w1);
                switch (a.k) {
                    case prog::K_CILKSORT: prog::warp_sort(a.p2, a.p0, a.p1, a.z1); break;   // src -> arr, tmp scratch
                    case prog::K_CILKMERGE: prog::warp_merge(a.p0, a.z1, a.p1, a.q1, a.p2); break;   // a, b -> dst
                    case prog::K_MERGESORT: prog::warp_sort(a.p0, a.p1, a.p2, a.z1); break;   // in -> out, tmp scratch
                    default: break;
                }
            }
            int* out = buf + (size_t)nbuf * prog::kLeafKeys;
            while (batch_of) {
                unsigned grp = 0;
                for (int c = 0; c < nbuf && batch_of; ++c) {
                    grp |= batch_of & (0u - batch_of);
                    batch_of &= batch_of - 1;
                }
                __syncwarp();   // the input buffers' previous contents are no longer read
                int j = 0;
                for (unsigned g = grp; g; g &= g - 1, ++j) {
                    const LeafArgs a = leaf_args(__ffs(g) - 1, kind, w0, w1);
                    int* in = buf + (size_t)j * prog::kLeafKeys;
                    if (a.k == prog::K_CILKSORT) prog::leaf_issue(a.p2, a.z1, a.p2, a.z1, in);
                    else if (a.k == prog::K_CILKMERGE) prog::leaf_issue(a.p0, a.z1, a.p1, a.z1 + a.q1, in);
                    else prog::leaf_issue(a.p0, a.z1, a.p0, a.z1, in);
                }
                prog::cp_async_wait_all();
                __syncwarp();
                j = 0;
                for (unsigned g = grp; g; g &= g - 1, ++j) {
                    const LeafArgs a = leaf_args(__ffs(g) - 1, kind, w0, w1);
                    int* in = buf + (size_t)j * prog::kLeafKeys;
                    if (a.k == prog::K_CILKSORT) prog::leaf_sort_out(in, a.z1, out, a.p0);
                    else if (a.k == prog::K_CILKMERGE) prog::leaf_merge_out(in, a.z1, a.q1, out, a.p2);
                    else prog::leaf_sort_out(in, a.z1, out, a.p1);
                }
            }
        } else {
            (void)A;
            (void)S;
            (void)mask;
            (void)kind;
            (void)w0;
            (void)w1;
        }
    }

    // w0/w1: the first 32 frame bytes, loaded together with the header
    __device__ static void exec(const Arena& A, WarpShared& S, int kind, int tid, void* frame, const int4& w0,
                                const int4& w1, unsigned long long fn) {
        (void)tid;
        (void)fn;
        switch (kind) {
            case prog::K_FIB: prog::fib_task<!kSorts && !kGraphs>(A, S, frame, w0); break;
            case prog::K_NQ: prog::nq_task(A, S, frame, w0); break;
            case prog::K_CILKSORT:
                if (kSorts) prog::cilksort_task(A, S, frame, w0, w1);
                else { GTAP_ERROR(A, ERR_INVALID_KIND, tid, -1, kind, 0); rt_finish(S); }
                break;
            case prog::K_CILKMERGE:
                if (kSorts) prog::cilkmerge_task(A, S, frame, w0, w1);
                else { GTAP_ERROR(A, ERR_INVALID_KIND, tid, -1, kind, 0); rt_finish(S); }
                break;
            case prog::K_MERGESORT:
                if (kSorts) prog::mergesort_task(A, S, frame, w0, w1);
                else { GTAP_ERROR(A, ERR_INVALID_KIND, tid, -1, kind, 0); rt_finish(S); }
                break;
            case prog::K_BFS:
                if constexpr (kGraphs) prog::bfs_task(A, S, frame, w0);
                else { GTAP_ERROR(A, ERR_INVALID_KIND, tid, -1, kind, 0); rt_finish(S); }
                break;
            case prog::K_TREESUM:
                if constexpr (kGraphs) prog::treesum_task(A, S, frame, w0, w1);
                else { GTAP_ERROR(A, ERR_INVALID_KIND, tid, -1, kind, 0); rt_finish(S); }
                break;
            default:
                GTAP_ERROR(A, ERR_INVALID_KIND, tid, -1, kind, 0);
                rt_finish(S);
                break;
        }
    }
};

using BuiltinProgram = BuiltinProgramT<true>;
using BuiltinProgramLight = BuiltinProgramT<false>;
using BuiltinProgramFibNq = BuiltinProgramT<false, false>;

}  // namespace gtap
