"""ctypes loader for the CPU oracle (oracle/liboracle.so).  Test infrastructure:
the product never imports this module."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

_L = None


def load():
    global _L
    if _L is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", ORACLE_DIR, os.path.join(ORACLE_DIR, "liboracle.so")], check=True,
                           capture_output=True)
        L = ctypes.CDLL(ORACLE_SO)
        i64, i32, u32, u64, vp = ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
        sig = {
            "orc_mt19937_fill_i32": (None, [u32, vp, i64]),
            "orc_mt19937_64_fill": (None, [u64, vp, i64]),
            "orc_fib": (i64, [ctypes.c_int]),
            "orc_fib_tasks": (i64, [ctypes.c_int, ctypes.c_int]),
            "orc_fib_executions": (i64, [ctypes.c_int, ctypes.c_int]),
            "orc_nq": (i64, [ctypes.c_int]),
            "orc_nq_tasks": (i64, [ctypes.c_int, ctypes.c_int]),
            "orc_sort_i32": (None, [vp, i64]),
            "orc_cilksort": (None, [vp, vp, i64, ctypes.c_int, ctypes.c_int, vp, vp]),
            "orc_mergesort_tasks": (i64, [i64, ctypes.c_int]),
            "orc_rmat_csr": (None, [ctypes.c_int, ctypes.c_int, u64, vp, vp]),
            "orc_max_degree_vertex": (i32, [vp, i32]),
            "orc_bfs": (None, [vp, vp, i32, i32, vp]),
            "orc_tree_gen": (None, [i32, u64, vp, vp, vp, vp]),
            "orc_tree_sum": (i64, [vp, vp, vp, i32]),
            "orc_root_mix": (None, [u64, i32, vp, vp, vp]),
            "orc_seq_root": (i64, [ctypes.c_int, ctypes.c_int, u64]),
            "orc_seq_cilksort": (None, [vp, vp, i64]),
            "orc_fmix32": (u32, [u32]),
            "orc_bary_input": (None, [u64, vp, i64]),
            "orc_bary_node_work": (u32, [u32, vp, i64, ctypes.c_int, ctypes.c_int]),
            "orc_bary_tree": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, i64, vp, vp]),
            "orc_bary_node_work_block": (u32, [u32, vp, i64, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "orc_bary_tree_block": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, i64,
                                           vp, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _L = L
    return _L


def p(a):
    return ctypes.c_void_p(a.ctypes.data)


def fib(n):
    return load().orc_fib(n)


def fib_tasks(n, cutoff=0):
    return load().orc_fib_tasks(n, cutoff)


def fib_executions(n, cutoff=0):
    return load().orc_fib_executions(n, cutoff)


def nq(n):
    return load().orc_nq(n)


def nq_tasks(n, cutoff_depth):
    return load().orc_nq_tasks(n, cutoff_depth)


def keys(seed, n):
    out = np.empty(n, np.int32)
    load().orc_mt19937_fill_i32(seed, p(out), n)
    return out


def mt64(seed, n):
    out = np.empty(n, np.uint64)
    load().orc_mt19937_64_fill(seed, p(out), n)
    return out


def sort(a):
    b = np.array(a, dtype=np.int32, copy=True)
    load().orc_sort_i32(p(b), len(b))
    return b


def cilksort(a, sort_cutoff, merge_cutoff):
    arr = np.array(a, dtype=np.int32, copy=True)
    tmp = np.empty_like(arr)
    st, mt = ctypes.c_int64(0), ctypes.c_int64(0)
    load().orc_cilksort(p(arr), p(tmp), len(arr), sort_cutoff, merge_cutoff, ctypes.byref(st), ctypes.byref(mt))
    return arr, st.value, mt.value


def mergesort_tasks(n, cutoff):
    return load().orc_mergesort_tasks(n, cutoff)


def rmat(scale, edge_factor=16, seed=42):
    nv = 1 << scale
    row = np.empty(nv + 1, np.int32)
    col = np.empty(nv * edge_factor, np.int32)
    load().orc_rmat_csr(scale, edge_factor, seed, p(row), p(col))
    return row, col


def max_degree_vertex(row):
    return load().orc_max_degree_vertex(p(row), len(row) - 1)


def bfs(row, col, src):
    nv = len(row) - 1
    depth = np.empty(nv, np.int32)
    load().orc_bfs(p(row), p(col), nv, src, p(depth))
    return depth


def tree(n, seed=42):
    left = np.empty(n, np.int32)
    right = np.empty(n, np.int32)
    value = np.empty(n, np.int32)
    size = np.empty(n, np.int32)
    load().orc_tree_gen(n, seed, p(left), p(right), p(value), p(size))
    return left, right, value, size


def tree_sum(left, right, value, root=0):
    return load().orc_tree_sum(p(left), p(right), p(value), root)


def root_mix(seed, n):
    kind = np.empty(n, np.int32)
    param = np.empty(n, np.int32)
    ks = np.empty(n, np.uint64)
    load().orc_root_mix(seed, n, p(kind), p(param), p(ks))
    return kind, param, ks


def bary_input(seed, n):
    out = np.empty(n, dtype=np.float64)
    load().orc_bary_input(seed, p(out), n)
    return out


def bary_tree(depth_max, branch, mem_ops, iters, inp):
    """(sum of the nodes' 32-bit mixes mod 2^64, node count) of the probabilistic B-ary tree."""
    s = np.zeros(1, dtype=np.uint64)
    c = np.zeros(1, dtype=np.int64)
    load().orc_bary_tree(depth_max, branch, mem_ops, iters, p(inp), len(inp), p(s), p(c))
    return int(s[0]), int(c[0])


def bary_tree_block(depth_max, branch, mem_ops, iters, threads, inp):
    """bary_tree with each node's work split over a block of `threads` threads."""
    s = np.zeros(1, dtype=np.uint64)
    c = np.zeros(1, dtype=np.int64)
    load().orc_bary_tree_block(depth_max, branch, mem_ops, iters, threads, p(inp), len(inp), p(s), p(c))
    return int(s[0]), int(c[0])
