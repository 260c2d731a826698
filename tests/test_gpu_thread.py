"""Parity of the thread-executed runtime against the CPU oracle (B200 only).

Every case runs through the C ABI (gtap_launch / gtap_launch_per_root /
gtap_run_host).  Integer results must be bit-exact; task counts must equal the
oracle's spawn-tree counts.  torch is used only to hold device buffers.
"""
import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    import torch
    torch.cuda.init()
    gt.gtap_initialize(gt.default_config())
    yield gt
    gt.gtap_finalize()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def dptr(t):
    return t.data_ptr()


def run1(root):
    res, st = gt.launch([root])
    return res[0], st


@pytest.mark.parametrize("n", [0, 1, 2, 3, 10, 20, 25, 30])
def test_fib_cutoff0(rt, n):
    r, st = run1(gt.fib_root(n))
    assert r.status == gt.ROOT_DONE
    assert r.value == orc.fib(n)
    assert r.tasks == orc.fib_tasks(n, 0)
    assert st.counters[0] == orc.fib_tasks(n, 0)            # tasks created
    # every task body runs once, every continuation once: as an execution of
    # its own, or at its join by the child that completes it (fib's sum)
    assert st.counters[1] + st.counters[10] == orc.fib_executions(n, 0)


def test_fib34_cutoff12(rt):
    r, st = run1(gt.fib_root(34, cutoff=12))
    assert r.value == 5702887
    assert r.tasks == orc.fib_tasks(34, 12) == 150049


@pytest.mark.parametrize("n", [1, 4, 6, 8, 10, 12, 13])
def test_nq_one_task_per_row(rt, n):
    r, st = run1(gt.nq_root(n))
    assert r.value == orc.nq(n)
    assert r.tasks == orc.nq_tasks(n, n - 1)


@pytest.mark.parametrize("n,cut", [(13, 7), (12, 3), (11, 0)])
def test_nq_reference_cutoff(rt, n, cut):
    r, st = run1(gt.nq_root(n, cut))
    assert r.value == orc.nq(n)
    assert r.tasks == orc.nq_tasks(n, cut)


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 1000, 4096, 1 << 16, (1 << 20) + 7])
def test_cilksort_thread(rt, n):
    import torch
    keys = orc.keys(42, n)
    src = dev(keys)
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    r, st = run1(gt.cilksort_root(dptr(src), dptr(arr), dptr(tmp), n, 64, 256))
    out = arr.cpu().numpy()
    assert np.array_equal(out, np.sort(keys))
    _, sort_tasks, merge_tasks = orc.cilksort(keys, 64, 256)
    assert r.tasks == sort_tasks + merge_tasks
    assert np.array_equal(src.cpu().numpy(), keys)    # input left untouched


@pytest.mark.parametrize("n", [1, 100, 129, 1 << 16, (1 << 20) + 3])
def test_mergesort_thread(rt, n):
    import torch
    keys = orc.keys(43, n)
    src = dev(keys)
    out = torch.empty_like(src)
    tmp = torch.empty_like(src)
    r, st = run1(gt.mergesort_root(dptr(src), dptr(out), dptr(tmp), n, 128, 256))
    assert np.array_equal(out.cpu().numpy(), np.sort(keys))


# Leaves of any length: sort cutoffs beyond one 64-key run and merge cutoffs
# beyond one 256-output tile go through the warp's run-and-merge passes.
@pytest.mark.parametrize("n,sc,mc", [(1 << 16, 2048, 2048), (100003, 1000, 700), (5000, 6000, 6000),
                                     ((1 << 20) + 1, 129, 257)])
def test_cilksort_large_leaves(rt, n, sc, mc):
    import torch
    keys = orc.keys(7, n)
    src = dev(keys)
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    r, st = run1(gt.cilksort_root(dptr(src), dptr(arr), dptr(tmp), n, sc, mc))
    assert r.status == gt.ROOT_DONE
    assert np.array_equal(arr.cpu().numpy(), np.sort(keys))
    _, sort_tasks, merge_tasks = orc.cilksort(keys, sc, mc)
    assert r.tasks == sort_tasks + merge_tasks


@pytest.mark.parametrize("n,cutoff", [(1 << 16, 1000), (77777, 4096), (300, 300)])
def test_mergesort_large_leaves(rt, n, cutoff):
    import torch
    keys = orc.keys(11, n)
    src = dev(keys)
    out = torch.empty_like(src)
    tmp = torch.empty_like(src)
    r, st = run1(gt.mergesort_root(dptr(src), dptr(out), dptr(tmp), n, cutoff, 256))
    assert r.status == gt.ROOT_DONE
    assert np.array_equal(out.cpu().numpy(), np.sort(keys))


def test_cilksort_duplicate_heavy_keys(rt):
    import torch
    rng = np.random.default_rng(3)
    keys = rng.integers(-3, 4, size=(1 << 18) + 5).astype(np.int32)
    keys[::97] = np.iinfo(np.int32).max
    keys[::89] = np.iinfo(np.int32).min
    src = dev(keys)
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    r, st = run1(gt.cilksort_root(dptr(src), dptr(arr), dptr(tmp), len(keys), 64, 256))
    assert np.array_equal(arr.cpu().numpy(), np.sort(keys))


@pytest.mark.parametrize("scale", [8, 12, 16])
def test_bfs_rmat(rt, scale):
    import torch
    row, col = gt.gen_rmat(scale, 16, 42)
    src = gt.max_degree_vertex(row)
    depth = torch.full((len(row) - 1,), 0x3f3f3f3f, dtype=torch.int32, device="cuda")
    drow, dcol = dev(row), dev(col)    # keep the device buffers alive during the launch
    r, st = run1(gt.bfs_root(dptr(drow), dptr(dcol), dptr(depth), len(row) - 1, src, 32))
    assert np.array_equal(depth.cpu().numpy(), orc.bfs(row, col, src))


@pytest.mark.parametrize("n,cutoff", [(1, 32), (1000, 1), (1 << 16, 32), (1 << 18, 64)])
def test_treesum(rt, n, cutoff):
    left, right, value, size = gt.gen_tree(n, 5)
    d = [dev(x) for x in (left, right, value, size)]
    r, st = run1(gt.treesum_root(*[dptr(x) for x in d], n, 0, cutoff))
    assert r.value == orc.tree_sum(left, right, value, 0)


# Serial leaves deeper than any earlier cutoff: the leaves are loops with a
# bounded stack of their own, so their depth does not depend on the device's
# per-thread stack size.
@pytest.mark.parametrize("n,cutoff", [(30, 31), (32, 20), (33, 16)])
def test_fib_deep_serial_leaves(rt, n, cutoff):
    r, st = run1(gt.fib_root(n, cutoff=cutoff))
    assert r.status == gt.ROOT_DONE
    assert r.value == orc.fib(n)
    assert r.tasks == orc.fib_tasks(n, cutoff)


@pytest.mark.parametrize("n,cut", [(14, 0), (12, 1), (8, 0)])
def test_nq_deep_serial_leaves(rt, n, cut):
    r, st = run1(gt.nq_root(n, cut))
    assert r.value == orc.nq(n)
    assert r.tasks == orc.nq_tasks(n, cut)


@pytest.mark.parametrize("cutoff", [65, 5000, 1 << 16])
def test_treesum_large_cutoff(rt, cutoff):
    # subtrees above 64 nodes take the size-guided walk (smaller child first)
    n = 1 << 16
    left, right, value, size = gt.gen_tree(n, 9)
    d = [dev(x) for x in (left, right, value, size)]
    r, st = run1(gt.treesum_root(*[dptr(x) for x in d], n, 0, cutoff))
    assert r.status == gt.ROOT_DONE
    assert r.value == orc.tree_sum(left, right, value, 0)


def mixed_roots(keep):
    import torch
    roots, expect, bufs = [], [], []
    for n in (5, 18, 22):
        roots.append(gt.fib_root(n))
        expect.append(("v", orc.fib(n)))
    for n in (6, 9):
        roots.append(gt.nq_root(n))
        expect.append(("v", orc.nq(n)))
    for n in (777, 1 << 14):
        keys = orc.keys(n, n)
        src = dev(keys)
        arr = torch.empty_like(src)
        tmp = torch.empty_like(src)
        keep += [src, arr, tmp]
        roots.append(gt.cilksort_root(dptr(src), dptr(arr), dptr(tmp), n))
        expect.append(("sorted", (arr, np.sort(keys))))
    return roots, expect


def check(results, expect):
    for r, (k, e) in zip(results, expect):
        assert r.status == gt.ROOT_DONE
        if k == "v":
            assert r.value == e
        else:
            arr, ref = e
            assert np.array_equal(arr.cpu().numpy(), ref)


def test_batch_mixed_one_launch(rt):
    keep = []
    roots, expect = mixed_roots(keep)
    res, st = gt.launch(roots)
    check(res, expect)
    assert sum(r.tasks for r in res) == st.counters[0]


def test_per_root_baseline_same_results(rt):
    keep = []
    roots, expect = mixed_roots(keep)
    res, st = gt.launch(roots, per_root=True)
    check(res, expect)


def test_batch_many_small_roots(rt):
    roots = [gt.fib_root(10 + (i % 9)) for i in range(3000)] + [gt.nq_root(8)] * 50
    res, st = gt.launch(roots)
    for r, root in zip(res, roots):
        assert r.status == gt.ROOT_DONE
        assert r.value == (orc.fib(root.i0) if root.kind == gt.KIND_FIB else 92)
        assert r.tasks == (orc.fib_tasks(root.i0, 0) if root.kind == gt.KIND_FIB else orc.nq_tasks(8, 7))
        assert r.t_done_ns >= r.t_admit_ns > 0


def test_run_host_buffers(rt):
    n = 50000
    keys = orc.keys(11, n)
    out = np.zeros(n, np.int32)
    tmp = np.zeros(n, np.int32)
    root = gt.cilksort_root(keys.ctypes.data, out.ctypes.data, tmp.ctypes.data, n)
    res, st, hin, hout = gt.run_host([root, gt.fib_root(20)])
    assert np.array_equal(out, np.sort(keys))
    assert res[1].value == 6765
    assert hin >= n * 4 and hout >= n * 4


def test_reset_then_relaunch(rt):
    gt.gtap_reset()
    r, _ = run1(gt.fib_root(24))
    assert r.value == orc.fib(24)
    assert gt.gtap_get_runtime_error_code() == 0


# ---- scheduler variants (still bit-exact) ------------------------------------
@pytest.mark.parametrize("kw", [
    dict(block=32), dict(block=1024), dict(steal_batch=1), dict(steal_batch=8),
    dict(victim_policy=gt.VICTIM_RANDOM, probe_width=1), dict(victim_policy=gt.VICTIM_LAST_SUCCESS),
    dict(num_queues=2), dict(num_queues=4), dict(deque_capacity=64), dict(grid=1, block=32),
    dict(admit_batch=32),
])
def test_variants(kw):
    gt.gtap_initialize(gt.default_config(**kw))
    try:
        r, st = run1(gt.fib_root(23))
        assert r.value == orc.fib(23) and r.tasks == orc.fib_tasks(23, 0)
        r, st = run1(gt.nq_root(10))
        assert r.value == 724
    finally:
        gt.gtap_finalize()


def test_overflow_queue_path():
    # tiny deques force the global overflow queue
    gt.gtap_initialize(gt.default_config(deque_capacity=64, grid=2, block=64))
    try:
        r, st = run1(gt.nq_root(11))
        assert r.value == 2680
        assert st.counters[9] > 0   # overflow pushes happened
    finally:
        gt.gtap_finalize()


def test_epaq_fib_three_queues():
    # evaluation/3-epaq/fib/fib_queue_3.cu: leaves on queue 1, continuations on queue 2
    gt.gtap_initialize(gt.default_config(num_queues=4))
    try:
        r, st = run1(gt.fib_root(30, cutoff=13, epaq=True))
        assert r.value == 832040 and r.tasks == orc.fib_tasks(30, 13)
    finally:
        gt.gtap_finalize()


@pytest.mark.parametrize("join_walk", [1, 8, 32])
def test_fib_sums_at_their_joins(join_walk):
    """gtap_config.join_walk: in rounds of at most join_walk tasks, the child
    that completes a fib task's join runs the task's sum and walks on to the
    ancestors whose joins that completes.  Values and task counts stay the
    oracle's; every continuation runs once, as an execution or at its join
    (with 32 every round walks, so every sum runs at its join).  Batches mix
    roots, so walks from different roots share rounds."""
    gt.gtap_initialize(gt.default_config(join_walk=join_walk))
    try:
        for n, cutoff in ((2, 0), (20, 0), (30, 0), (34, 12)):
            r, st = run1(gt.fib_root(n, cutoff))
            assert r.status == gt.ROOT_DONE and r.value == orc.fib(n)
            assert r.tasks == orc.fib_tasks(n, cutoff)
            assert st.counters[1] + st.counters[10] == orc.fib_executions(n, cutoff)
            if join_walk == 32:
                assert st.counters[10] == orc.fib_executions(n, cutoff) - orc.fib_tasks(n, cutoff)
        roots = [gt.fib_root(18 + i % 11) for i in range(64)] + [gt.nq_root(8 + i % 4) for i in range(64)]
        res, st = gt.launch(roots)
        for i, r in enumerate(res[:64]):
            n = 18 + i % 11
            assert r.status == gt.ROOT_DONE and r.value == orc.fib(n) and r.tasks == orc.fib_tasks(n, 0)
        for i, r in enumerate(res[64:]):
            n = 8 + i % 4
            assert r.value == orc.nq(n) and r.tasks == orc.nq_tasks(n, n - 1)
    finally:
        gt.gtap_finalize()
    # EPAQ: the walk ignores the continuation's queue, results do not change
    gt.gtap_initialize(gt.default_config(num_queues=4, join_walk=join_walk))
    try:
        r, st = run1(gt.fib_root(30, cutoff=13, epaq=True))
        assert r.value == 832040 and r.tasks == orc.fib_tasks(30, 13)
    finally:
        gt.gtap_finalize()


@pytest.mark.parametrize("sub_rounds", [1, 8])
def test_sub_rounds_on_idle_lanes(sub_rounds):
    """gtap_config.sub_rounds: a round with idle lanes runs more passes of task
    bodies on them over the children staged in the round.  Values, task
    counts and executions stay the oracle's, alone and with the join walk,
    for single roots (whose ramp-up and drain leave lanes idle) and for a
    batch of fib and n-queens roots."""
    for join_walk in (0, 32):
        gt.gtap_initialize(gt.default_config(sub_rounds=sub_rounds, join_walk=join_walk))
        try:
            for n, cutoff in ((1, 0), (2, 0), (20, 0), (30, 0), (34, 12)):
                r, st = run1(gt.fib_root(n, cutoff))
                assert r.status == gt.ROOT_DONE and r.value == orc.fib(n)
                assert r.tasks == orc.fib_tasks(n, cutoff)
                assert st.counters[1] + st.counters[10] == orc.fib_executions(n, cutoff)
            for n in (1, 8, 12, 13):
                r, st = run1(gt.nq_root(n))
                assert r.value == orc.nq(n) and r.tasks == orc.nq_tasks(n, n - 1)
            r, st = run1(gt.nq_root(13, 7))
            assert r.value == orc.nq(13) and r.tasks == orc.nq_tasks(13, 7)
            roots = [gt.fib_root(18 + i % 11) for i in range(48)] + [gt.nq_root(8 + i % 4) for i in range(48)]
            res, st = gt.launch(roots)
            for i, r in enumerate(res[:48]):
                n = 18 + i % 11
                assert r.status == gt.ROOT_DONE and r.value == orc.fib(n) and r.tasks == orc.fib_tasks(n, 0)
            for i, r in enumerate(res[48:]):
                n = 8 + i % 4
                assert r.value == orc.nq(n) and r.tasks == orc.nq_tasks(n, n - 1)
        finally:
            gt.gtap_finalize()
