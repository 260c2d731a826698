"""Admission orders on the device (B200 only): a batch of all six built-in
kinds, interleaved, gives the same values, task counts, sorted bytes and BFS
depths under GTAP_ADMIT_AS_GIVEN, GTAP_ADMIT_BY_KIND and GTAP_ADMIT_SPLIT, with
results in the caller's order (results[i].index == i), and each checked
against the oracle.  A split batch whose first launch fails (an unknown kind,
the kernel's own check) reports the error and leaves the sorts pending."""
import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

INF = 0x3f3f3f3f


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


class Batch:
    """Interleaved fib / n-queens / cilksort / mergesort / BFS / tree-sum roots."""

    def __init__(self):
        import torch
        self.roots, self.checks, self.keep, self.depths = [], [], [], []
        rng = np.random.default_rng(7)
        row, col = gt.gen_rmat(11, 16, 77)
        self.bfs_src = gt.max_degree_vertex(row)
        self.bfs_want = orc.bfs(row, col, self.bfs_src)
        self.drow, self.dcol = dev(row), dev(col)
        tree = gt.gen_tree(5000, 3)
        self.tree_want = orc.tree_sum(*tree[:3], 0)
        self.dtree = [dev(x) for x in tree]
        for i in range(60):
            k = i % 6
            if k == 0:
                n = int(rng.integers(10, 23))
                self.roots.append(gt.fib_root(n))
                self.checks.append(("fib", n))
            elif k == 1:
                n = int(rng.integers(6, 10))
                self.roots.append(gt.nq_root(n))
                self.checks.append(("nq", n))
            elif k in (2, 3):
                n = int(rng.integers(1000, 70000))
                keys = orc.keys(500 + i, n)
                src = dev(keys)
                out, tmp = torch.empty_like(src), torch.empty_like(src)
                self.keep += [src, out, tmp]
                mk = gt.cilksort_root if k == 2 else gt.mergesort_root
                self.roots.append(mk(src.data_ptr(), out.data_ptr(), tmp.data_ptr(), n))
                self.checks.append(("sort", (out, np.sort(keys))))
            elif k == 4:
                depth = torch.full((len(row) - 1,), INF, dtype=torch.int32, device="cuda")
                self.depths.append(depth)
                self.roots.append(gt.bfs_root(self.drow.data_ptr(), self.dcol.data_ptr(), depth.data_ptr(),
                                              len(row) - 1, self.bfs_src))
                self.checks.append(("bfs", depth))
            else:
                self.roots.append(gt.treesum_root(*[x.data_ptr() for x in self.dtree], 5000, 0, 32))
                self.checks.append(("tree", None))

    def run(self):
        for d in self.depths:
            d.fill_(INF)
        for k, c in self.checks:
            if k == "sort":
                c[0].zero_()
        return gt.launch(self.roots)

    def check(self, res):
        bad = []
        for i, (r, (k, c)) in enumerate(zip(res, self.checks)):
            if r.status != gt.ROOT_DONE or r.index != i:
                bad.append((i, "status/index", r.status, r.index))
            elif k == "fib" and (r.value, r.tasks) != (orc.fib(c), orc.fib_tasks(c, 0)):
                bad.append((i, k, c, r.value, r.tasks))
            elif k == "nq" and (r.value, r.tasks) != (orc.nq(c), orc.nq_tasks(c, c - 1)):
                bad.append((i, k, c, r.value, r.tasks))
            elif k == "sort" and not np.array_equal(c[0].cpu().numpy(), c[1]):
                bad.append((i, k))
            elif k == "bfs" and not np.array_equal(c.cpu().numpy(), self.bfs_want):
                bad.append((i, k))
            elif k == "tree" and r.value != self.tree_want:
                bad.append((i, k, r.value))
        assert not bad, bad[:10]


@pytest.fixture(scope="module")
def batch():
    import torch
    torch.cuda.init()
    return Batch()


def test_every_admission_order_gives_the_same_results(batch):
    seen = {}
    for order, launches in ((gt.ADMIT_AS_GIVEN, 1), (gt.ADMIT_BY_KIND, 1), (gt.ADMIT_SPLIT, 2)):
        gt.gtap_initialize(gt.default_config(admit_order=order))
        try:
            res, st = batch.run()
        finally:
            gt.gtap_finalize()
        assert st.status == 0
        assert st.launches == launches
        assert sum(r.tasks for r in res) == st.counters[0]
        batch.check(res)
        if order == gt.ADMIT_SPLIT:
            assert 0 < st.light_kernel_ms < st.kernel_ms and st.light_workers > 0
        # an asynchronous BFS may relax a vertex more than once: its task count is not fixed
        seen[order] = [(r.value, -1 if k == "bfs" else r.tasks, r.status, r.index)
                       for r, (k, _) in zip(res, batch.checks)]
    assert seen[gt.ADMIT_AS_GIVEN] == seen[gt.ADMIT_BY_KIND] == seen[gt.ADMIT_SPLIT]


def test_split_batch_with_a_failing_first_launch(batch):
    gt.gtap_initialize(gt.default_config())
    try:
        roots = [batch.roots[2], gt.Root(kind=99), gt.fib_root(12)]
        arr = (gt.Root * 3)(*roots)
        res = (gt.RootResult * 3)()
        st = gt.RunStats()
        rc = gt.lib().gtap_launch(arr, 3, res, gt.ctypes.byref(st), None)
        assert rc == 10, rc                  # unknown task kind, raised by the first launch
        assert st.launches == 1 and st.status == 10
        assert res[0].status == gt.ROOT_PENDING and res[0].index == 0   # the sort never ran
        assert [r.index for r in res] == [0, 1, 2]
        res2, st2 = gt.launch([gt.fib_root(15), batch.roots[2]])
        assert res2[0].value == 610 and st2.launches == 2
    finally:
        gt.gtap_finalize()


@pytest.mark.parametrize("pinned", [True, False])
def test_host_buffer_batch_in_three_launches(pinned):
    """gtap_run_host: sort roots slicing one host buffer (one copy each way),
    one sort with buffers of its own, fib / n-queens / BFS / tree-sum roots
    around them.  The roots other than sorts run in two launches, one on each
    side of the sort launch; every output matches the oracle."""
    import torch
    torch.cuda.init()
    rng = np.random.default_rng(3)
    sizes = [int(x) for x in rng.integers(500, 40000, size=24)]
    total = sum(sizes)
    keys = orc.keys(91, total)

    def host(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.pin_memory() if pinned else t

    src, out = host(keys), host(np.zeros(total, np.int32))
    lone_keys = orc.keys(92, 12345)
    lone_src, lone_out = host(lone_keys), host(np.zeros(12345, np.int32))
    row, col = gt.gen_rmat(10, 16, 5)
    bsrc = gt.max_degree_vertex(row)
    hrow, hcol = host(row), host(col)
    depth = host(np.full(len(row) - 1, INF, np.int32))
    tree = [host(x) for x in gt.gen_tree(3000, 9)]
    roots, want = [], []
    off = 0
    for i, n in enumerate(sizes):
        roots.append(gt.cilksort_root(src.data_ptr() + 4 * off, out.data_ptr() + 4 * off, 0, n))
        want.append(("sort", None))
        roots.append(gt.fib_root(12 + i % 8) if i % 2 == 0 else gt.nq_root(6 + i % 3))
        want.append(("fib", 12 + i % 8) if i % 2 == 0 else ("nq", 6 + i % 3))
        off += n
    roots.insert(5, gt.cilksort_root(lone_src.data_ptr(), lone_out.data_ptr(), 0, 12345))
    want.insert(5, ("sort", None))
    roots.append(gt.bfs_root(hrow.data_ptr(), hcol.data_ptr(), depth.data_ptr(), len(row) - 1, bsrc))
    want.append(("bfs", None))
    roots.append(gt.treesum_root(*[t.data_ptr() for t in tree], 3000, 0, 32))
    want.append(("tree", None))

    gt.gtap_initialize(gt.default_config())
    try:
        res, st, hin, hout = gt.run_host(roots)
    finally:
        gt.gtap_finalize()
    assert st.status == 0 and st.launches == 3
    for i, (r, (k, p)) in enumerate(zip(res, want)):
        assert r.status == gt.ROOT_DONE and r.index == i
        if k == "fib":
            assert (r.value, r.tasks) == (orc.fib(p), orc.fib_tasks(p, 0))
        elif k == "nq":
            assert (r.value, r.tasks) == (orc.nq(p), orc.nq_tasks(p, p - 1))
    off = 0
    for n in sizes:
        assert np.array_equal(out.numpy()[off:off + n], np.sort(keys[off:off + n]))
        off += n
    assert np.array_equal(lone_out.numpy(), np.sort(lone_keys))
    assert np.array_equal(depth.numpy(), orc.bfs(row, col, bsrc))
    assert res[-1].value == orc.tree_sum(*[t.numpy() for t in tree[:3]], 0)
    # every input array once, every output array once, and the root tables
    in_bytes = 4 * (total + 12345) + row.nbytes + col.nbytes + depth.numpy().nbytes + 4 * 4 * 3000
    assert hin == in_bytes + 56 * len(roots)
    assert hout == 4 * (total + 12345) + depth.numpy().nbytes + 40 * len(roots)
