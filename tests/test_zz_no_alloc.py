"""gtap_launch_noalloc: running roots without allocating device memory (B200 only).

Some callers of this library cannot call cudaMalloc: a serving loop that must
not take the device-wide synchronisation an allocation can cause, or a process
whose device memory already belongs to another allocator (a framework pool
holding nearly all of HBM, where a new cudaMalloc fails or fragments).  For
them gtap_launch_noalloc keeps the scheduler's working memory in a fixed
device array inside the library; the caller only supplies device buffers for
the root descriptors, the results and the arrays the roots read.

This test calls it through the C ABI twice in a row and checks every result
against the regular entry point gtap_launch on the same roots (integer results
must match exactly), and that device free memory does not move across a call
once the one-time set-up has happened.  The file name makes pytest collect it
last.
"""
import ctypes

import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

INF = 0x3f3f3f3f


def _device_bytes(struct_array):
    import torch
    raw = bytes(memoryview(struct_array).cast("B"))
    return torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()


def _results_from_device(t, n):
    raw = t.cpu().numpy().tobytes()
    out = (gt.RootResult * n)()
    ctypes.memmove(out, raw, ctypes.sizeof(out))
    return list(out)


def test_noalloc_matches_gtap_launch_twice():
    import torch
    torch.cuda.init()
    # inputs owned by the caller: a tree and an R-MAT graph on the device
    left, right, value, size = gt.gen_tree(1 << 16, 5)
    tree = [torch.from_numpy(x).cuda() for x in (left, right, value, size)]
    row, col = gt.gen_rmat(12, 16, 42)
    src = gt.max_degree_vertex(row)
    drow, dcol = torch.from_numpy(row).cuda(), torch.from_numpy(col).cuda()
    nv = len(row) - 1
    depth_ref = torch.full((nv,), INF, dtype=torch.int32, device="cuda")
    depth_na = torch.full((nv,), INF, dtype=torch.int32, device="cuda")

    def roots(depth):
        # about 260k tasks in all, well inside the 2^19 records the scratch holds
        return [gt.fib_root(24), gt.fib_root(30, cutoff=12), gt.fib_root(32, cutoff=14), gt.nq_root(10), gt.nq_root(12, 4),
                gt.treesum_root(*[x.data_ptr() for x in tree], 1 << 16, 0, 32),
                gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), depth.data_ptr(), nv, src, 32)]

    # the regular entry point (allocates its arena in gtap_initialize)
    gt.gtap_initialize(gt.default_config())
    try:
        ref, _ = gt.launch(roots(depth_ref))
    finally:
        gt.gtap_finalize()
    assert all(r.status == gt.ROOT_DONE for r in ref)
    assert ref[1].value == 832040 and ref[3].value == 724
    assert [r.tasks for r in ref[:5]] == [orc.fib_tasks(24), orc.fib_tasks(30, 12), orc.fib_tasks(32, 14),
                                          orc.nq_tasks(10, 9), orc.nq_tasks(12, 4)]
    want_depth = orc.bfs(row, col, src)
    assert np.array_equal(depth_ref.cpu().numpy(), want_depth)

    # the allocation-free entry point: descriptors and results live in device
    # buffers the caller allocated up front
    rs = roots(depth_na)
    arr = (gt.Root * len(rs))(*rs)
    d_roots = _device_bytes(arr)
    d_results = torch.zeros(ctypes.sizeof(gt.RootResult) * len(rs), dtype=torch.uint8, device="cuda")
    free_before = None
    for call in range(2):
        depth_na.fill_(INF)
        torch.cuda.synchronize()
        if call == 1:
            free_before = torch.cuda.mem_get_info()[0]
        rc = gt.lib().gtap_launch_noalloc(ctypes.c_void_p(d_roots.data_ptr()), len(rs),
                                          ctypes.c_void_p(d_results.data_ptr()), None)
        assert rc == 0, gt.gtap_get_runtime_error_string(rc)
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before   # nothing was allocated
        got = _results_from_device(d_results, len(rs))
        for i, (a, b) in enumerate(zip(got, ref)):
            assert a.status == gt.ROOT_DONE
            assert a.value == b.value
            # an asynchronous BFS spawns one task per successful relaxation, a
            # number that depends on timing; every other root's count is fixed
            if rs[i].kind != gt.KIND_BFS:
                assert a.tasks == b.tasks
        assert np.array_equal(depth_na.cpu().numpy(), want_depth)


def _noalloc_call(roots):
    import torch
    arr = (gt.Root * len(roots))(*roots)
    d_roots = _device_bytes(arr)
    d_results = torch.zeros(ctypes.sizeof(gt.RootResult) * len(roots), dtype=torch.uint8, device="cuda")
    rc = gt.lib().gtap_launch_noalloc(ctypes.c_void_p(d_roots.data_ptr()), len(roots),
                                      ctypes.c_void_p(d_results.data_ptr()), None)
    return rc, (_results_from_device(d_results, len(roots)) if rc == 0 else None)


def _small_roots_exact():
    roots = [gt.fib_root(20), gt.fib_root(26, cutoff=10), gt.nq_root(9)]
    rc, got = _noalloc_call(roots)
    assert rc == 0, gt.gtap_get_runtime_error_string(rc)
    assert [r.value for r in got] == [orc.fib(20), orc.fib(26), orc.nq(9)]
    assert [r.tasks for r in got] == [orc.fib_tasks(20), orc.fib_tasks(26, 10), orc.nq_tasks(9, 8)]


def test_noalloc_after_gtap_initialize_with_a_small_block():
    """gtap_initialize sets the shared-memory limit of the same worker kernel
    from its own configuration; a 32-thread block with a small staging buffer
    lowers it below what the allocation-free entry point launches with.  The
    entry point sets its limit on every call, so it keeps working."""
    import torch
    torch.cuda.init()
    _small_roots_exact()
    gt.gtap_initialize(gt.default_config(block=32, spawn_capacity=64))
    gt.gtap_finalize()
    _small_roots_exact()
    _small_roots_exact()


def test_noalloc_reports_an_outgrown_scratch_and_recovers():
    """A tree whose live tasks outgrow the 2^19 records of the scratch array
    ends with GTAP_ERROR_TASK_ID_POOL_LOW_HEADROOM, a status the kernel
    returns, not a fault; the next call starts from a clean scratch and is
    exact.  n-queens(16) with every row forking is such a tree: each task
    creates all of its children at once (up to 16), so some ten rounds of
    every worker running 32 tasks hold far more than 2^19 ready tasks.
    (A fib tree keeps its live set small: fib(34) without a cutoff fits.)"""
    import torch
    torch.cuda.init()
    rc, _ = _noalloc_call([gt.nq_root(16, 15)])
    assert rc == 6, rc
    _small_roots_exact()


def test_noalloc_rejects_too_many_roots():
    import torch
    torch.cuda.init()
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    assert gt.lib().gtap_launch_noalloc(ctypes.c_void_p(d.data_ptr()), 4097, ctypes.c_void_p(d.data_ptr()),
                                        None) == gt.ERROR_INVALID_ARGUMENT
    assert gt.lib().gtap_launch_noalloc(None, 1, None, None) == gt.ERROR_INVALID_ARGUMENT
