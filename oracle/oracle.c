/*
 * oracle.c -- CPU restatement of the GTaP workloads (TEST INFRASTRUCTURE ONLY).
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker; the gtap_b200 product never links or calls it.  Each function
 * cites the reference file:line it restates; declarations are in oracle.h.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* MT19937 / MT19937-64 (Matsumoto & Nishimura), restated from the papers.  */
/* ------------------------------------------------------------------------ */
typedef struct { uint32_t mt[624]; int idx; } mt32_t;

static void mt32_seed(mt32_t* s, uint32_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
}

static uint32_t mt32_next(mt32_t* s) {
    if (s->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            uint32_t v = s->mt[(i + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
            s->mt[i] = v;
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

typedef struct { uint64_t mt[312]; int idx; } mt64_t;

static void mt64_seed(mt64_t* s, uint64_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        s->mt[i] = 6364136223846793005ull * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
    s->idx = 312;
}

static uint64_t mt64_next(mt64_t* s) {
    if (s->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            uint64_t x = (s->mt[i] & 0xFFFFFFFF80000000ull) | (s->mt[(i + 1) % 312] & 0x7FFFFFFFull);
            uint64_t v = s->mt[(i + 156) % 312] ^ (x >> 1);
            if (x & 1ull) v ^= 0xB5026F5AA96619E9ull;
            s->mt[i] = v;
        }
        s->idx = 0;
    }
    uint64_t x = s->mt[s->idx++];
    x ^= (x >> 29) & 0x5555555555555555ull;
    x ^= (x << 17) & 0x71D67FFFEDA60000ull;
    x ^= (x << 37) & 0xFFF7EEE000000000ull;
    x ^= x >> 43;
    return x;
}

void orc_mt19937_fill_i32(uint32_t seed, int32_t* out, int64_t n) {
    mt32_t s;
    mt32_seed(&s, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = (int32_t)mt32_next(&s);
}

void orc_mt19937_64_fill(uint64_t seed, uint64_t* out, int64_t n) {
    mt64_t* s = (mt64_t*)malloc(sizeof(mt64_t));
    mt64_seed(s, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = mt64_next(s);
    free(s);
}

/* ------------------------------------------------------------------------ */
/* fib                                                                      */
/* ------------------------------------------------------------------------ */
/* evaluation/2-comparison/fib/seq_fib.c:5-10 */
int64_t orc_fib(int n) {
    if (n < 2) return n;
    int64_t a = 0, b = 1;            /* iterative form of the same recurrence */
    for (int i = 1; i < n; ++i) { int64_t c = a + b; a = b; b = c; }
    return b;
}

/* gtap_fib.cu:10-22 / fib_queue_1.cu:16-26: task(n) spawns task(n-1) and
 * task(n-2) unless n < max(cutoff, 2). */
static int leaf_below(int cutoff) { return cutoff < 2 ? 2 : cutoff; }

int64_t orc_fib_tasks(int n, int cutoff) {
    int c = leaf_below(cutoff);
    /* T(n) = 1 for n < c, T(n) = 1 + T(n-1) + T(n-2) otherwise. */
    int64_t t[128];
    if (n < 0 || n >= 128) return -1;
    for (int i = 0; i <= n; ++i)
        t[i] = (i < c) ? 1 : 1 + t[i - 1] + t[i - 2];
    return t[n];
}

int64_t orc_fib_executions(int n, int cutoff) {
    /* every non-leaf task executes twice (spawn, then resume after taskwait) */
    int c = leaf_below(cutoff);
    int64_t t[128];
    if (n < 0 || n >= 128) return -1;
    for (int i = 0; i <= n; ++i)
        t[i] = (i < c) ? 1 : 2 + t[i - 1] + t[i - 2];
    return t[n];
}

/* ------------------------------------------------------------------------ */
/* n-queens                                                                 */
/* ------------------------------------------------------------------------ */
/* evaluation/2-comparison/nq/seq_nq.c:13-34 (same bit tricks as gtap_nq.cu:10-23) */
static int64_t nq_solve(int row, uint32_t column, uint32_t left, uint32_t right, int n) {
    if (row == n) return 1;
    uint32_t mask = (n < 32 ? (1u << n) - 1u : 0xFFFFFFFFu);
    uint32_t avail = mask & ~(column | left | right);
    int64_t total = 0;
    while (avail) {
        uint32_t p = avail & (0u - avail);
        avail -= p;
        total += nq_solve(row + 1, column | p, (left | p) << 1, (right | p) >> 1, n);
    }
    return total;
}

int64_t orc_nq(int n) { return nq_solve(0, 0, 0, 0, n); }

/* gtap_nq.cu:25-55: tasks at row <= cutoff fork per free column. */
static int64_t nq_tasks(int row, uint32_t column, uint32_t left, uint32_t right, int n, int cutoff) {
    if (row > cutoff) return 1;          /* runs serial_search, spawns nothing */
    uint32_t mask = (n < 32 ? (1u << n) - 1u : 0xFFFFFFFFu);
    uint32_t avail = mask & ~(column | left | right);
    int64_t total = 1;
    while (avail) {
        uint32_t p = avail & (0u - avail);
        avail -= p;
        total += nq_tasks(row + 1, column | p, (left | p) << 1, (right | p) >> 1, n, cutoff);
    }
    return total;
}

int64_t orc_nq_tasks(int n, int cutoff_depth) { return nq_tasks(0, 0, 0, 0, n, cutoff_depth); }

/* ------------------------------------------------------------------------ */
/* sorting                                                                  */
/* ------------------------------------------------------------------------ */
void orc_sort_i32(int32_t* a, int64_t n) {
    if (n < 2) return;
    uint32_t* src = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    uint32_t* dst = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) src[i] = (uint32_t)a[i] ^ 0x80000000u;
    for (int pass = 0; pass < 4; ++pass) {
        int64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        int sh = pass * 8;
        for (int64_t i = 0; i < n; ++i) cnt[((src[i] >> sh) & 0xFF) + 1]++;
        for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
        for (int64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xFF]++] = src[i];
        uint32_t* t = src; src = dst; dst = t;
    }
    for (int64_t i = 0; i < n; ++i) a[i] = (int32_t)(src[i] ^ 0x80000000u);
    free(src);
    free(dst);
}

static int cmp_i32(const void* x, const void* y) {
    int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
    return (a > b) - (a < b);
}

/* examples/cilksort/cilksort.cu:17-36 (merge_device) */
static void seq_merge(const int32_t* a, int64_t an, const int32_t* b, int64_t bn, int32_t* dst) {
    int64_t i = 0, j = 0, k = 0;
    while (i < an && j < bn) {
        if (a[i] < b[j]) dst[k++] = a[i++];
        else dst[k++] = b[j++];
    }
    while (i < an) dst[k++] = a[i++];
    while (j < bn) dst[k++] = b[j++];
}

/* examples/cilksort/cilksort.cu:38-49: largest index with x[idx] <= val */
static int64_t bsearch_le(const int32_t* x, int64_t len, int32_t val) {
    int64_t low = -1, high = len;
    while (low + 1 < high) {
        int64_t mid = (low + high) / 2;
        if (x[mid] <= val) low = mid; else high = mid;
    }
    return low;
}

/* examples/cilksort/cilksort.cu:89-125 */
static void cilkmerge_rec(const int32_t* a, int64_t an, const int32_t* b, int64_t bn,
                          int32_t* dst, int cutoff, int64_t* tasks) {
    ++*tasks;
    if (an < bn) {
        const int32_t* t = a; a = b; b = t;
        int64_t tn = an; an = bn; bn = tn;
    }
    if (bn == 0) {
        if (an > 0) memcpy(dst, a, sizeof(int32_t) * (size_t)an);
        return;
    }
    if (an + bn < cutoff) {
        seq_merge(a, an, b, bn, dst);
        return;
    }
    int64_t as = (an + 1) / 2;
    int64_t bs = bsearch_le(b, bn, a[as - 1]) + 1;
    cilkmerge_rec(a, as, b, bs, dst, cutoff, tasks);
    cilkmerge_rec(a + as, an - as, b + bs, bn - bs, dst + as + bs, cutoff, tasks);
}

/* examples/cilksort/cilksort.cu:127-164 */
static void cilksort_rec(int32_t* arr, int64_t n, int32_t* tmp, int sort_cutoff,
                         int merge_cutoff, int64_t* st, int64_t* mt) {
    ++*st;
    if (n < sort_cutoff) {
        qsort(arr, (size_t)n, sizeof(int32_t), cmp_i32);
        return;
    }
    int64_t len12 = n / 2, len1 = len12 / 2, len2 = len12 - len1;
    int64_t len34 = n - len12, len3 = len34 / 2, len4 = len34 - len3;
    cilksort_rec(arr, len1, tmp, sort_cutoff, merge_cutoff, st, mt);
    cilksort_rec(arr + len1, len2, tmp + len1, sort_cutoff, merge_cutoff, st, mt);
    cilksort_rec(arr + len12, len3, tmp + len12, sort_cutoff, merge_cutoff, st, mt);
    cilksort_rec(arr + len12 + len3, len4, tmp + len12 + len3, sort_cutoff, merge_cutoff, st, mt);
    cilkmerge_rec(arr, len1, arr + len1, len2, tmp, merge_cutoff, mt);
    cilkmerge_rec(arr + len12, len3, arr + len12 + len3, len4, tmp + len12, merge_cutoff, mt);
    cilkmerge_rec(tmp, len12, tmp + len12, len34, arr, merge_cutoff, mt);
}

void orc_cilksort(int32_t* arr, int32_t* tmp, int64_t n, int sort_cutoff,
                  int merge_cutoff, int64_t* sort_tasks, int64_t* merge_tasks) {
    int64_t st = 0, mt = 0;
    cilksort_rec(arr, n, tmp, sort_cutoff, merge_cutoff, &st, &mt);
    if (sort_tasks) *sort_tasks = st;
    if (merge_tasks) *merge_tasks = mt;
}

/* examples/mergesort/mergesort.cu:34-50 */
int64_t orc_mergesort_tasks(int64_t n, int cutoff) {
    if (n <= 1) return 1;
    if (n <= cutoff) return 1;
    int64_t left = (n + 1) / 2;          /* [left, mid] holds ceil(n/2) */
    return 1 + orc_mergesort_tasks(left, cutoff) + orc_mergesort_tasks(n - left, cutoff);
}

/* ------------------------------------------------------------------------ */
/* R-MAT + BFS                                                              */
/* ------------------------------------------------------------------------ */
static int cmp_u64(const void* x, const void* y) {
    uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
    return (a > b) - (a < b);
}

void orc_rmat_csr(int scale, int edge_factor, uint64_t seed, int32_t* row, int32_t* col) {
    int64_t nv = (int64_t)1 << scale;
    int64_t ne = nv * edge_factor;
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)ne);
    mt64_t* s = (mt64_t*)malloc(sizeof(mt64_t));
    mt64_seed(s, seed);
    for (int64_t e = 0; e < ne; ++e) {
        uint64_t src = 0, dst = 0;
        for (int lvl = 0; lvl < scale; ++lvl) {
            uint64_t r = mt64_next(s) % 100;
            uint64_t sb = 0, db = 0;
            if (r < 57) { sb = 0; db = 0; }
            else if (r < 76) { sb = 0; db = 1; }
            else if (r < 95) { sb = 1; db = 0; }
            else { sb = 1; db = 1; }
            src = (src << 1) | sb;
            dst = (dst << 1) | db;
        }
        keys[e] = (src << 32) | dst;
    }
    free(s);
    qsort(keys, (size_t)ne, sizeof(uint64_t), cmp_u64);
    memset(row, 0, sizeof(int32_t) * (size_t)(nv + 1));
    for (int64_t e = 0; e < ne; ++e) {
        row[(keys[e] >> 32) + 1]++;
        col[e] = (int32_t)(keys[e] & 0xFFFFFFFFu);
    }
    for (int64_t v = 0; v < nv; ++v) row[v + 1] += row[v];
    free(keys);
}

int32_t orc_max_degree_vertex(const int32_t* row, int32_t nv) {
    int32_t best = 0, bd = -1;
    for (int32_t v = 0; v < nv; ++v) {
        int32_t d = row[v + 1] - row[v];
        if (d > bd) { bd = d; best = v; }
    }
    return best;
}

/* examples/asynchronous_bfs/asynchronous_bfs_thread.cu:143-175 */
void orc_bfs(const int32_t* row, const int32_t* col, int32_t nv, int32_t src, int32_t* depth) {
    const int32_t INF = 0x3f3f3f3f;
    for (int32_t i = 0; i < nv; ++i) depth[i] = INF;
    int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)nv);
    int64_t head = 0, tail = 0;
    depth[src] = 0;
    q[tail++] = src;
    while (head < tail) {
        int32_t v = q[head++];
        int32_t dv = depth[v];
        for (int32_t e = row[v]; e < row[v + 1]; ++e) {
            int32_t u = col[e];
            if (dv + 1 < depth[u]) {
                depth[u] = dv + 1;
                q[tail++] = u;
            }
        }
    }
    free(q);
}

/* ------------------------------------------------------------------------ */
/* tree sum                                                                 */
/* ------------------------------------------------------------------------ */
void orc_tree_gen(int32_t n, uint64_t seed, int32_t* left, int32_t* right,
                  int32_t* value, int32_t* size) {
    mt64_t* s = (mt64_t*)malloc(sizeof(mt64_t));
    mt64_seed(s, seed);
    int32_t* pl = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);   /* preorder arrays */
    int32_t* pr = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* pv = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* ps = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* sb = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);   /* stack: budgets */
    int32_t* si = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);   /* stack: positions */
    int32_t sp = 0, next = 0;
    sb[sp] = n; si[sp] = next++; ++sp;
    while (sp > 0) {
        --sp;
        int32_t b = sb[sp], i = si[sp];
        pv[i] = (int32_t)(uint32_t)mt64_next(s);
        int32_t L = 0;
        for (int32_t k = 0; k < b - 1; ++k)
            if (mt64_next(s) % 100 < 48) ++L;
        int32_t R = b - 1 - L;
        ps[i] = b;
        pl[i] = L > 0 ? i + 1 : -1;
        pr[i] = R > 0 ? i + 1 + L : -1;
        /* preorder: left subtree occupies [i+1, i+1+L), right [i+1+L, i+b) */
        if (R > 0) { sb[sp] = R; si[sp] = i + 1 + L; ++sp; }
        if (L > 0) { sb[sp] = L; si[sp] = i + 1; ++sp; }
        (void)next;
    }
    /* seeded relabelling, root kept at 0 */
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    for (int32_t i = 0; i < n; ++i) perm[i] = i;
    for (int32_t i = n - 1; i >= 2; --i) {
        int32_t j = 1 + (int32_t)(mt64_next(s) % (uint64_t)i);   /* j in [1, i] */
        int32_t t = perm[i]; perm[i] = perm[j]; perm[j] = t;
    }
    for (int32_t i = 0; i < n; ++i) {
        int32_t p = perm[i];
        left[p] = pl[i] >= 0 ? perm[pl[i]] : -1;
        right[p] = pr[i] >= 0 ? perm[pr[i]] : -1;
        value[p] = pv[i];
        size[p] = ps[i];
    }
    free(perm); free(pl); free(pr); free(pv); free(ps); free(sb); free(si); free(s);
}

int64_t orc_tree_sum(const int32_t* left, const int32_t* right, const int32_t* value, int32_t root) {
    /* iterative preorder walk; the count of nodes bounds the stack */
    int64_t cap = 1024, sp = 0, total = 0;
    int32_t* st = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    st[sp++] = root;
    while (sp > 0) {
        int32_t v = st[--sp];
        total += value[v];
        if (sp + 2 > cap) { cap *= 2; st = (int32_t*)realloc(st, sizeof(int32_t) * (size_t)cap); }
        if (left[v] >= 0) st[sp++] = left[v];
        if (right[v] >= 0) st[sp++] = right[v];
    }
    free(st);
    return total;
}

/* ------------------------------------------------------------------------ */
/* batched root mix                                                         */
/* ------------------------------------------------------------------------ */
void orc_root_mix(uint64_t seed, int32_t n_roots, int32_t* kind, int32_t* param, uint64_t* key_seed) {
    mt64_t* s = (mt64_t*)malloc(sizeof(mt64_t));
    mt64_seed(s, seed);
    for (int32_t i = 0; i < n_roots; ++i) {
        uint64_t d0 = mt64_next(s), d1 = mt64_next(s), d2 = mt64_next(s);
        int32_t k = (int32_t)(d0 % 3);
        kind[i] = k;
        if (k == 0) param[i] = 18 + (int32_t)(d1 % 11);
        else if (k == 1) param[i] = 8 + (int32_t)(d1 % 4);
        else param[i] = (int32_t)((1024 + (d1 >> 8) % 1024) << (d1 % 10));
        key_seed[i] = d2;
    }
    free(s);
}

/* ------------------------------------------------------------------------ */
/* sequential CPU baseline                                                  */
/* ------------------------------------------------------------------------ */
/* evaluation/2-comparison/fib/seq_fib.c:5-10 */
static int seq_fib_rec(int n) {
    if (n < 2) return n;
    return seq_fib_rec(n - 1) + seq_fib_rec(n - 2);
}

/* evaluation/2-comparison/cilksort/seq_cilksort.cpp:38-48 */
static void seq_merge_le(const int32_t* a, int64_t an, const int32_t* b, int64_t bn, int32_t* dst) {
    int64_t i = 0, j = 0, k = 0;
    while (i < an && j < bn) {
        if (a[i] <= b[j]) dst[k++] = a[i++];
        else dst[k++] = b[j++];
    }
    while (i < an) dst[k++] = a[i++];
    while (j < bn) dst[k++] = b[j++];
}

/* evaluation/2-comparison/cilksort/seq_cilksort.cpp:50-69 */
static void seq_cilksort_rec(int32_t* arr, int32_t* tmp, int64_t n) {
    if (n < 2) return;
    int64_t n12 = n / 2, n1 = n12 / 2, n2 = n12 - n1;
    int64_t n34 = n - n12, n3 = n34 / 2, n4 = n34 - n3;
    seq_cilksort_rec(arr, tmp, n1);
    seq_cilksort_rec(arr + n1, tmp + n1, n2);
    seq_cilksort_rec(arr + n12, tmp + n12, n3);
    seq_cilksort_rec(arr + n12 + n3, tmp + n12 + n3, n4);
    seq_merge_le(arr, n1, arr + n1, n2, tmp);
    seq_merge_le(arr + n12, n3, arr + n12 + n3, n4, tmp + n12);
    seq_merge_le(tmp, n12, tmp + n12, n34, arr);
}

void orc_seq_cilksort(int32_t* arr, int32_t* tmp, int64_t n) { seq_cilksort_rec(arr, tmp, n); }

int64_t orc_seq_root(int kind, int param, uint64_t seed) {
    if (kind == 0) return seq_fib_rec(param);
    if (kind == 1) return nq_solve(0, 0, 0, 0, param);
    int64_t n = param;
    int32_t* a = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* t = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    orc_mt19937_fill_i32((uint32_t)seed, a, n);
    seq_cilksort_rec(a, t, n);
    int64_t ok = 1;
    for (int64_t i = 1; i < n; ++i)
        if (a[i - 1] > a[i]) { ok = 0; break; }
    free(a);
    free(t);
    return ok;
}

/* ---- probabilistic B-ary tree (gtap_thread_tree_load_compute.cu:96-143) -- */
uint32_t orc_fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

void orc_bary_input(uint64_t seed, double* out, int64_t n) {
    uint64_t x = seed;
    for (int64_t i = 0; i < n; ++i) {
        x += 0x9e3779b97f4a7c15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        out[i] = (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
}

uint32_t orc_bary_node_work(uint32_t node, const double* input, int64_t n, int mem_ops, int iters) {
    const uint32_t seed = orc_fmix32(node ^ 0x2545f491u);
    double acc = 0.0;
    for (int m = 0; m < mem_ops; ++m) acc += input[orc_fmix32(seed + (uint32_t)m) & (uint32_t)(n - 1)];
    uint32_t mix = (seed ^ 0x9e3779b9u) + (uint32_t)(int32_t)acc;
    double y = 0.0;
    for (int it = 0; it < iters; ++it) {
        const double x = (double)orc_fmix32(seed + (uint32_t)it * 0x632be5abu);
        y = fma(x, 1.0000001192092896, y);
        uint64_t bits;
        memcpy(&bits, &y, sizeof(bits));
        mix ^= (uint32_t)bits ^ (uint32_t)(bits >> 32);
    }
    return mix;
}

uint32_t orc_bary_node_work_block(uint32_t node, const double* input, int64_t n, int mem_ops, int iters, int threads) {
    const uint32_t seed = orc_fmix32(node ^ 0x2545f491u);
    double acc = 0.0;
    uint32_t xr = 0;
    for (int t = 0; t < threads; ++t) {
        double part = 0.0;
        for (int m = t; m < mem_ops; m += threads) part += input[orc_fmix32(seed + (uint32_t)m) & (uint32_t)(n - 1)];
        acc += part;
        double y = 0.0;
        for (int it = t; it < iters; it += threads) {
            const double x = (double)orc_fmix32(seed + (uint32_t)it * 0x632be5abu);
            y = fma(x, 1.0000001192092896, y);
            uint64_t bits;
            memcpy(&bits, &y, sizeof(bits));
            xr ^= (uint32_t)bits ^ (uint32_t)(bits >> 32);
        }
    }
    return ((seed ^ 0x9e3779b9u) + (uint32_t)(int32_t)acc) ^ xr;
}

/* threads == 0: thread mode (orc_bary_node_work), else block mode with that many threads */
static void bary_rec(uint32_t node, int d, int D, int B, int mem_ops, int iters, int threads, const double* input,
                     int64_t n, uint64_t* sum, int64_t* nodes) {
    if (d < D) {
        uint32_t s = orc_fmix32(node ^ ((uint32_t)d * 0x9e3779b9u));
        for (int k = 0; k < B; ++k) {
            s = orc_fmix32(s + (uint32_t)k);
            if ((int)(s % (uint32_t)D) < D - d)
                bary_rec(node * (uint32_t)B + (uint32_t)(k + 1), d + 1, D, B, mem_ops, iters, threads, input, n, sum,
                         nodes);
        }
    }
    *sum += threads ? orc_bary_node_work_block(node, input, n, mem_ops, iters, threads)
                    : orc_bary_node_work(node, input, n, mem_ops, iters);
    *nodes += 1;
}

void orc_bary_tree(int depth_max, int branch, int mem_ops, int iters, const double* input, int64_t n,
                   uint64_t* sum, int64_t* nodes) {
    *sum = 0;
    *nodes = 0;
    bary_rec(0u, 0, depth_max, branch, mem_ops, iters, 0, input, n, sum, nodes);
}

void orc_bary_tree_block(int depth_max, int branch, int mem_ops, int iters, int threads, const double* input,
                         int64_t n, uint64_t* sum, int64_t* nodes) {
    *sum = 0;
    *nodes = 0;
    bary_rec(0u, 0, depth_max, branch, mem_ops, iters, threads < 1 ? 1 : threads, input, n, sum, nodes);
}
