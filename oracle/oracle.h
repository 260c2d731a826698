/*
 * oracle.h -- CPU restatement of the GTaP workloads and of their spawn trees.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the gtap_b200 product links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker (or as the timed CPU baseline).
 *
 * Every function cites the reference file:line whose algorithm it restates
 * (paths are relative to the reference project root).  Parity is pinned by
 * tests/test_oracle.py against (a) the reference's own sequential programs,
 * compiled from their sources into oracle/_ref/ by oracle/Makefile and run on
 * the same inputs, and (b) the known answers recorded in tests/golden/.
 */
#ifndef GTAP_ORACLE_H
#define GTAP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- pseudo random generators (published algorithms) ------------------- */
/* MT19937, Matsumoto & Nishimura 1998; equals C++ std::mt19937(seed). */
void orc_mt19937_fill_i32(uint32_t seed, int32_t* out, int64_t n);
/* MT19937-64, Nishimura 2000; equals C++ std::mt19937_64(seed). */
void orc_mt19937_64_fill(uint64_t seed, uint64_t* out, int64_t n);

/* ---- fib: evaluation/2-comparison/fib/seq_fib.c:5-10 --------------------- */
int64_t orc_fib(int n);
/* Spawned-task count of the fib task tree (root included):
 * gtap_fib.cu:10-22 (cutoff <= 2) and evaluation/3-epaq/fib/fib_queue_1.cu:16-26
 * (a task with n < cutoff runs fib_sequential and spawns nothing). */
int64_t orc_fib_tasks(int n, int cutoff);
/* Executions (task tasks plus continuations resumed after taskwait). */
int64_t orc_fib_executions(int n, int cutoff);

/* ---- n-queens: evaluation/2-comparison/nq/seq_nq.c:13-34 ----------------- */
int64_t orc_nq(int n);
/* Task count for gtap_nq.cu:25-55: a task at row <= cutoff_depth spawns one
 * child per free column; a task at row > cutoff_depth runs serial_search.
 * "One task per row" is cutoff_depth = n-1 (row-n tasks count a solution). */
int64_t orc_nq_tasks(int n, int cutoff_depth);

/* ---- sorting ------------------------------------------------------------ */
/* Ascending int32 sort (LSD radix); output equals std::sort. */
void orc_sort_i32(int32_t* a, int64_t n);
/* The cilksort recursion of examples/cilksort/cilksort.cu:89-164 with its
 * sort/merge spawn cutoffs as parameters; sorts arr in place using tmp and
 * returns the number of cilksort and cilkmerge tasks (root included). */
void orc_cilksort(int32_t* arr, int32_t* tmp, int64_t n, int sort_cutoff,
                  int merge_cutoff, int64_t* sort_tasks, int64_t* merge_tasks);
/* Task count of examples/mergesort/mergesort.cu:34-50 (cutoff 128 there):
 * a task with n > cutoff spawns two halves, otherwise sorts serially. */
int64_t orc_mergesort_tasks(int64_t n, int cutoff);

/* ---- BFS: examples/asynchronous_bfs/asynchronous_bfs_thread.cu:143-175 ---- */
/* R-MAT edge list -> CSR sorted by (src,dst).  row has 2^scale+1 entries,
 * col has edge_factor*2^scale entries.  Quadrant probabilities (percent):
 * a=57 b=19 c=19 d=5, one mt19937_64 draw per level (draw % 100). */
void orc_rmat_csr(int scale, int edge_factor, uint64_t seed, int32_t* row,
                  int32_t* col);
/* Vertex of maximum out-degree, lowest id on ties. */
int32_t orc_max_degree_vertex(const int32_t* row, int32_t nv);
/* Queue BFS; unreached vertices keep 0x3f3f3f3f (cudaMemset 0x3f). */
void orc_bfs(const int32_t* row, const int32_t* col, int32_t nv, int32_t src,
             int32_t* depth);
/* Number of tasks the asynchronous BFS would spawn is schedule dependent;
 * only the depth array is compared. */

/* ---- tree sum ----------------------------------------------------------- */
/* Random unbalanced binary tree of n nodes: a node with budget b sends each
 * of its b-1 descendants left with probability 48% (one mt19937_64 draw per
 * descendant, draw % 100 < 48).  Nodes are laid out in preorder and then
 * relabelled by a seeded Fisher-Yates permutation (root kept at 0).
 * left/right hold child ids or -1, value holds int32 payloads, size holds
 * subtree sizes. */
void orc_tree_gen(int32_t n, uint64_t seed, int32_t* left, int32_t* right,
                  int32_t* value, int32_t* size);
int64_t orc_tree_sum(const int32_t* left, const int32_t* right,
                     const int32_t* value, int32_t root);

/* ---- batched root mix --------------------------------------------------- */
/* kind[i]: 0 fib, 1 nq, 2 cilksort.  param[i]: fib n, nq n, or array size.
 * seed[i]: key seed (mt19937 of the low 32 bits).  Three mt19937_64 draws
 * per root: kind = d0 % 3; fib n = 18 + d1 % 11; nq n = 8 + d1 % 4;
 * cilksort size = (1024 + (d1 >> 8) % 1024) << (d1 % 10); seed = d2. */
void orc_root_mix(uint64_t seed, int32_t n_roots, int32_t* kind,
                  int32_t* param, uint64_t* key_seed);

/* ---- sequential CPU baseline of one mix root --------------------------- */
/* Runs one root the way the reference's sequential programs do:
 * kind 0: fib recursion of evaluation/2-comparison/fib/seq_fib.c:5-10;
 * kind 1: n-queens solve() of evaluation/2-comparison/nq/seq_nq.c:13-34;
 * kind 2: cilksort_rec/merge_seq of evaluation/2-comparison/cilksort/seq_cilksort.cpp:38-69
 *         on mt19937(seed) keys (sorted keys are checked, 1 = sorted).
 * Returns the root's value. */
int64_t orc_seq_root(int kind, int param, uint64_t seed);
/* seq_cilksort.cpp:50-69 on caller-provided keys (no key generation inside). */
void orc_seq_cilksort(int32_t* arr, int32_t* tmp, int64_t n);

/* ---- probabilistic B-ary tree ------------------------------------------- *
 * The workload shape of evaluation/2-comparison/prob_Bary_tree/
 * gtap_thread_tree_load_compute.cu:96-143: a node at depth d < D keeps each
 * of its B child candidates with probability 1 - d/D, drawn from a hash of
 * the node id; every node does seeded loads of a double array and a loop of
 * fused multiply-adds after its children finish.  Here each node's work ends
 * in a 32-bit mix that is summed over all nodes (a deterministic result, where
 * the reference's own program only stores into a racy sink).  Hash: the
 * MurmurHash3 32-bit finaliser; input: splitmix64 (Steele, Lea, Flood 2014)
 * mapped to doubles in [-1, 1). */
uint32_t orc_fmix32(uint32_t h);
void orc_bary_input(uint64_t seed, double* out, int64_t n);
uint32_t orc_bary_node_work(uint32_t node, const double* input, int64_t n, int mem_ops, int iters);
void orc_bary_tree(int depth_max, int branch, int mem_ops, int iters, const double* input, int64_t n,
                   uint64_t* sum, int64_t* nodes);
/* Block mode (gtap_block_tree_load_compute.cu): the same tree, each node's
 * work split over the T threads of a block -- thread t takes loads m = t,
 * t+T, ... and fma steps it = t, t+T, ... in order; the T partial sums are
 * added in thread order and the T xor-words combined. */
uint32_t orc_bary_node_work_block(uint32_t node, const double* input, int64_t n, int mem_ops, int iters, int threads);
void orc_bary_tree_block(int depth_max, int branch, int mem_ops, int iters, int threads, const double* input,
                         int64_t n, uint64_t* sum, int64_t* nodes);

#ifdef __cplusplus
}
#endif
#endif
