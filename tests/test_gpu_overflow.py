"""Detached children past the staging buffer (B200 only).

A task that spawns more detached children in one round than its warp's
staging buffer holds (BFS leaves over long edge ranges, n-queens rows) sends
the surplus to the global overflow queue.  Such a child becomes visible only
after the spawning task has written its frame, and its creation is counted for
its root before any other warp can run it.  These cases run with the smallest
staging buffer (64 entries) so that most children take that path, with several
roots of different sizes in one launch, so that a child run on a stale frame
would read another root's indices; every result must equal the oracle's.
"""
import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

INF = 0x3f3f3f3f


@pytest.fixture(scope="module")
def small_staging():
    import torch
    torch.cuda.init()
    gt.gtap_initialize(gt.default_config(spawn_capacity=64))
    yield gt
    gt.gtap_finalize()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("split", [64, 1024, 1 << 16])
def test_bfs_roots_of_three_sizes_in_one_launch(small_staging, split):
    import torch
    roots, keep, want = [], [], []
    for scale in (11, 14, 16):
        row, col = gt.gen_rmat(scale, 16, 300 + scale)
        src = gt.max_degree_vertex(row)
        drow, dcol = dev(row), dev(col)
        depth = torch.full((len(row) - 1,), INF, dtype=torch.int32, device="cuda")
        keep += [drow, dcol, depth]
        roots.append(gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), depth.data_ptr(), len(row) - 1, src, split))
        want.append((depth, orc.bfs(row, col, src)))
    res, st = gt.launch(roots)
    assert st.status == 0
    assert all(r.status == gt.ROOT_DONE for r in res)
    for depth, ref in want:
        assert np.array_equal(depth.cpu().numpy(), ref)
    assert st.as_dict()["overflow_pushes"] > 0       # the path under test ran
    assert sum(r.tasks for r in res) == st.counters[0]


def test_nq_every_row_forks(small_staging):
    # n-queens 12 with every row forking: up to 12 detached children per task
    res, st = gt.launch([gt.nq_root(12, 11), gt.nq_root(11, 10), gt.nq_root(10, 9)])
    assert st.status == 0
    assert [r.value for r in res] == [orc.nq(12), orc.nq(11), orc.nq(10)]
    assert [r.tasks for r in res] == [orc.nq_tasks(12, 11), orc.nq_tasks(11, 10), orc.nq_tasks(10, 9)]
    assert st.counters[0] == sum(r.tasks for r in res)


def test_mixed_kinds_share_the_overflow_queue(small_staging):
    import torch
    roots, keep, checks = [], [], []
    row, col = gt.gen_rmat(15, 16, 77)
    src = gt.max_degree_vertex(row)
    drow, dcol = dev(row), dev(col)
    keep += [drow, dcol]
    ref = orc.bfs(row, col, src)
    left, right, value, size = gt.gen_tree(1 << 17, 21)
    tree = [dev(x) for x in (left, right, value, size)]
    tsum = orc.tree_sum(left, right, value, 0)
    for i in range(12):
        k = i % 3
        if k == 0:
            depth = torch.full((len(row) - 1,), INF, dtype=torch.int32, device="cuda")
            keep.append(depth)
            roots.append(gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), depth.data_ptr(), len(row) - 1, src, 4096))
            checks.append(("bfs", depth))
        elif k == 1:
            roots.append(gt.treesum_root(*[t.data_ptr() for t in tree], 1 << 17, 0, 32))
            checks.append(("v", tsum))
        else:
            roots.append(gt.nq_root(10, 9))
            checks.append(("v", orc.nq(10)))
    res, st = gt.launch(roots)
    assert st.status == 0
    for r, (kind, want) in zip(res, checks):
        assert r.status == gt.ROOT_DONE
        if kind == "bfs":
            assert np.array_equal(want.cpu().numpy(), ref)
        else:
            assert r.value == want
    assert sum(r.tasks for r in res) == st.counters[0]
