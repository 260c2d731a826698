"""The global rings across the 2^32 wrap of their cursors (B200 only).

The overflow queue and the recycled-id pool keep their positions across
launches, and a slot's tag is the lap of its position (gtap_b200/csrc/
gtap_ring.h).  A long-lived process (a serving loop, repeated launches)
eventually wraps the 32-bit cursors.  These cases place both rings' cursors a
few dozen positions below the wrap with the testing aid
gtap_debug_set_ring_position, then run launches whose overflow traffic crosses
it, with the smallest staging buffer so that most detached children take the
overflow path; every result must equal the oracle's, on the launch that
crosses the wrap and on the launches after it.
"""
import ctypes

import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

INF = 0x3f3f3f3f
NEAR_WRAP = (1 << 32) - 48


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _roots(keep):
    """Four roots whose detached children overflow a 64-entry staging buffer,
    with their expected values (None: check the depth array in keep)."""
    import torch
    row, col = gt.gen_rmat(14, 16, 914)
    src = gt.max_degree_vertex(row)
    drow, dcol = _dev(row), _dev(col)
    depth = torch.full((len(row) - 1,), INF, dtype=torch.int32, device="cuda")
    keep += [drow, dcol, depth]
    roots = [gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), depth.data_ptr(), len(row) - 1, src, 1024),
             gt.nq_root(10, 9), gt.fib_root(22), gt.nq_root(9, 8)]
    want = [None, orc.nq(10), orc.fib(22), orc.nq(9)]
    return roots, want, depth, orc.bfs(row, col, src)


def test_rings_cross_the_cursor_wrap():
    import torch
    torch.cuda.init()
    gt.gtap_initialize(gt.default_config(spawn_capacity=64))
    try:
        keep = []
        roots, want, depth, want_depth = _roots(keep)
        gt.set_ring_position(NEAR_WRAP)
        pushes = 0
        for launch in range(3):
            depth.fill_(INF)
            res, st = gt.launch(roots)
            assert st.status == 0
            assert all(r.status == gt.ROOT_DONE for r in res)
            for r, w in zip(res, want):
                if w is not None:
                    assert r.value == w
            assert res[1].tasks == orc.nq_tasks(10, 9) and res[2].tasks == orc.fib_tasks(22)
            assert np.array_equal(depth.cpu().numpy(), want_depth)
            pushes += st.as_dict()["overflow_pushes"]
        # the overflow queue really moved past position 2^32 - 1
        assert pushes > (1 << 32) - NEAR_WRAP
    finally:
        gt.gtap_finalize()


def test_noalloc_rings_cross_the_cursor_wrap():
    """The same for gtap_launch_noalloc's scratch array.  Its staging buffer
    holds 512 children; BFS tasks over the long edge ranges of the graph's
    hub vertices spawn more, and every launch recycles ids through the pool."""
    import torch
    torch.cuda.init()
    keep = []
    roots, want, depth, want_depth = _roots(keep)
    arr = (gt.Root * len(roots))(*roots)
    d_roots = torch.frombuffer(bytearray(bytes(memoryview(arr).cast("B"))), dtype=torch.uint8).cuda()
    d_results = torch.zeros(ctypes.sizeof(gt.RootResult) * len(roots), dtype=torch.uint8, device="cuda")

    def call():
        depth.fill_(INF)
        torch.cuda.synchronize()
        rc = gt.lib().gtap_launch_noalloc(ctypes.c_void_p(d_roots.data_ptr()), len(roots),
                                          ctypes.c_void_p(d_results.data_ptr()), None)
        assert rc == 0, gt.gtap_get_runtime_error_string(rc)
        raw = d_results.cpu().numpy().tobytes()
        out = (gt.RootResult * len(roots))()
        ctypes.memmove(out, raw, ctypes.sizeof(out))
        for r, w in zip(out, want):
            assert r.status == gt.ROOT_DONE
            if w is not None:
                assert r.value == w
        assert out[1].tasks == orc.nq_tasks(10, 9) and out[2].tasks == orc.fib_tasks(22)
        assert np.array_equal(depth.cpu().numpy(), want_depth)

    call()                                  # the first call sets the device up
    gt.set_ring_position(NEAR_WRAP, target=1)
    for _ in range(3):
        call()
