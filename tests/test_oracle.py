"""The CPU oracle against the reference's own answers (CPU only).

Pins: tests/golden/known_answers.json (written by tests/golden/make_golden.py
from the reference's sequential programs) and, when oracle/_ref is built here,
the reference programs themselves on the same inputs.
"""
import hashlib
import json
import os
import re
import subprocess

import numpy as np
import pytest

from tests import oracle_lib as orc

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def test_fib_matches_reference_seq_fib():
    for n, v in GOLD["fib"].items():
        assert orc.fib(int(n)) == v


def test_fib_task_tree_counts():
    assert orc.fib_tasks(30, 0) == GOLD["fib_tasks"]["30_0"]
    assert orc.fib_tasks(34, 12) == GOLD["fib_tasks"]["34_12"]
    assert orc.fib_executions(30, 0) == GOLD["fib_executions"]["30_0"]
    # closed form of the cutoff-0 spawn tree: 2*fib(n+1) - 1
    for n in range(2, 25):
        assert orc.fib_tasks(n, 0) == 2 * orc.fib(n + 1) - 1


def test_nq_matches_reference_seq_nq():
    for n, v in GOLD["nq"].items():
        assert orc.nq(int(n)) == v


def test_nq_task_tree():
    assert orc.nq_tasks(13, 12) == GOLD["nq_tasks"]["13_12"]
    # the task tree at cutoff n-1 has one node per partial placement; its
    # leaves at row n are exactly the solutions
    for n in range(4, 10):
        assert orc.nq_tasks(n, n - 1) >= orc.nq(n)


def test_mt19937_known_answers():
    # C++ standard [rand.predef]: 10000th output of the default-seeded engines
    assert int(np.uint32(orc.keys(5489, 10000)[-1])) == GOLD["mt19937_seed5489_10000th"]
    assert int(orc.mt64(5489, 10000)[-1]) == GOLD["mt19937_64_seed5489_10000th"]


@pytest.mark.parametrize("n", [1 << 10, 1 << 16])
def test_keys_and_sort_digests(n):
    g = GOLD["sorts_seed42"][str(n)]
    k = orc.keys(42, n)
    assert [int(x) for x in k[:8]] == g["keys_first8"]
    assert hashlib.sha256(k.tobytes()).hexdigest() == g["keys_sha256"]
    assert hashlib.sha256(orc.sort(k).tobytes()).hexdigest() == g["sorted_sha256"]
    assert g["reference_seq_cilksort_correct"] and g["reference_seq_mergesort_correct"]


@pytest.mark.parametrize("n,sc,mc", [(0, 64, 256), (1, 64, 256), (63, 64, 256), (1000, 64, 256),
                                     (1 << 14, 64, 256), (99991, 2048, 2048)])
def test_cilksort_recursion_sorts(n, sc, mc):
    k = orc.keys(7, n)
    arr, st, mt = orc.cilksort(k, sc, mc)
    assert np.array_equal(arr, np.sort(k))
    assert st >= 1 and mt >= 0


def test_mergesort_task_count():
    # n <= cutoff: one task; otherwise 1 + halves
    assert orc.mergesort_tasks(128, 128) == 1
    assert orc.mergesort_tasks(129, 128) == 3
    assert orc.mergesort_tasks(1 << 24, 128) == 2 * (1 << 17) - 1


def test_bfs_against_scipy():
    sp = pytest.importorskip("scipy.sparse")
    csg = pytest.importorskip("scipy.sparse.csgraph")
    row, col = orc.rmat(10, 16, 42)
    src = orc.max_degree_vertex(row)
    d = orc.bfs(row, col, src)
    nv = len(row) - 1
    m = sp.csr_matrix((np.ones(len(col)), col, row), shape=(nv, nv))
    ref = csg.shortest_path(m, unweighted=True, indices=src, directed=True)
    ref = np.where(np.isinf(ref), 0x3f3f3f3f, ref).astype(np.int64)
    assert np.array_equal(d.astype(np.int64), ref)


def test_tree_shape_and_sum():
    n = 5000
    left, right, value, size = orc.tree(n, 3)
    # every node appears exactly once as a child except the root (node 0)
    kids = np.concatenate([left[left >= 0], right[right >= 0]])
    assert len(kids) == n - 1 and len(np.unique(kids)) == n - 1 and 0 not in kids
    assert size[0] == n
    assert orc.tree_sum(left, right, value, 0) == int(value.astype(np.int64).sum())


def test_root_mix_ranges():
    kind, param, ks = orc.root_mix(42, 4096)
    assert set(np.unique(kind)) <= {0, 1, 2}
    assert param[kind == 0].min() >= 18 and param[kind == 0].max() <= 28
    assert param[kind == 1].min() >= 8 and param[kind == 1].max() <= 11
    cs = param[kind == 2]
    assert cs.min() >= 1 << 10 and cs.max() < 1 << 20


REF = orc.REF_DIR


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "seq_nq")), reason="reference programs not built here")
def test_oracle_against_reference_programs_live():
    out = subprocess.run([os.path.join(REF, "seq_fib"), "27"], capture_output=True, text=True).stdout
    assert int(re.search(r"is (\d+)", out).group(1)) == orc.fib(27)
    out = subprocess.run([os.path.join(REF, "seq_nq"), "11"], capture_output=True, text=True).stdout
    assert int(re.search(r"= (\d+)", out).group(1)) == orc.nq(11)
