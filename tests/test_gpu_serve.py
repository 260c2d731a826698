"""Serve mode on the GPU (B200 only): a persistent kernel admits roots that the
host publishes while it runs.

Roots of every register-light kind (fib, n-queens, BFS on R-MAT graphs, tree
sums) are enqueued in waves, some before earlier ones have finished, polled
to completion, and checked against the oracle; ring slots are reused after
their roots were polled.  The ring refuses more unpolled roots than it
holds, and the kernel stops on shutdown.
"""
import time

import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

INF = 0x3f3f3f3f


@pytest.fixture(scope="module")
def graphs():
    import torch
    torch.cuda.init()
    out = []
    for scale in (10, 13):
        row, col = gt.gen_rmat(scale, 16, 42 + scale)
        src = gt.max_degree_vertex(row)
        out.append((row, col, src, torch.from_numpy(row).cuda(), torch.from_numpy(col).cuda(),
                    orc.bfs(row, col, src)))
    return out


def poll_all(pending, timeout_s=20.0):
    done = {}
    t0 = time.time()
    while pending and time.time() - t0 < timeout_s:
        for i in gt.serve_poll(1024):
            done[i] = True
            pending.discard(i)
    assert not pending, "roots not completed: %s" % sorted(pending)[:8]
    return done


def test_serve_waves_match_oracle(graphs):
    import torch
    left, right, value, size = gt.gen_tree(1 << 15, 3)
    tree = [torch.from_numpy(x).cuda() for x in (left, right, value, size)]
    tree_sum = orc.tree_sum(left, right, value, 0)
    # every device buffer exists before the session starts: while the
    # persistent kernel holds the SMs, no other kernel (a torch fill) may run
    nv_max = max(len(g[0]) - 1 for g in graphs)
    depths = [torch.full((nv_max,), INF, dtype=torch.int32, device="cuda") for _ in range(12)]
    torch.cuda.synchronize()
    gt.gtap_initialize(gt.default_config())
    try:
        gt.serve_start(ring_capacity=64)
        nb = 0
        expect = {}
        for wave in range(4):
            roots, kinds = [], []
            for j in range(12):
                k = (wave * 12 + j) % 4
                if k == 0:
                    n = 15 + (j % 8)
                    roots.append(gt.fib_root(n))
                    kinds.append(("v", orc.fib(n)))
                elif k == 1:
                    n = 6 + (j % 5)
                    roots.append(gt.nq_root(n))
                    kinds.append(("v", orc.nq(n)))
                elif k == 2:
                    row, col, src, drow, dcol, want = graphs[j % 2]
                    d = depths[nb]
                    nb += 1
                    roots.append(gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), d.data_ptr(), len(row) - 1, src, 32))
                    kinds.append(("bfs", (d, want)))
                else:
                    roots.append(gt.treesum_root(*[t.data_ptr() for t in tree], 1 << 15, 0, 32))
                    kinds.append(("v", tree_sum))
            first = gt.serve_enqueue(roots)
            for i, k in enumerate(kinds):
                expect[(first + i) % 64] = k
            # every second wave goes in while the previous one may still run;
            # then everything outstanding is polled and checked
            if wave % 2 == 1:
                poll_all(set(expect))
                slots = sorted(expect)
                for i, r in zip(slots, gt.serve_results(slots)):
                    kind, want = expect[i]
                    assert r.status == gt.ROOT_DONE
                    assert r.t_done_ns >= r.t_admit_ns > 0
                    if kind == "v":
                        assert r.value == want
                    else:
                        d, ref = want
                        assert np.array_equal(d.cpu().numpy()[:len(ref)], ref)
                expect = {}
        st = gt.serve_shutdown()
        assert st.status == 0
        assert st.counters[0] > 0
    finally:
        gt.gtap_finalize()


def test_serve_bfs_roots_past_the_staging_buffer():
    # the smallest staging buffer and BFS leaves over up to 4096 edges: most
    # children go through the overflow queue while roots keep arriving
    import torch
    torch.cuda.init()
    graphs = []
    for scale in (14, 16):
        row, col = gt.gen_rmat(scale, 16, 500 + scale)
        src = gt.max_degree_vertex(row)
        graphs.append((row, col, src, torch.from_numpy(row).cuda(), torch.from_numpy(col).cuda(),
                       orc.bfs(row, col, src)))
    left, right, value, size = gt.gen_tree(1 << 17, 8)
    tree = [torch.from_numpy(x).cuda() for x in (left, right, value, size)]
    tree_sum = orc.tree_sum(left, right, value, 0)
    depths = [torch.full((len(graphs[i % 2][0]) - 1,), INF, dtype=torch.int32, device="cuda") for i in range(24)]
    torch.cuda.synchronize()
    gt.gtap_initialize(gt.default_config(spawn_capacity=64))
    try:
        gt.serve_start(ring_capacity=64)
        expect = {}
        for wave in range(4):
            roots, kinds = [], []
            for j in range(8):
                i = wave * 6 + j
                if j < 6:
                    row, col, src, drow, dcol, want = graphs[i % 2]
                    d = depths[i]
                    roots.append(gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), d.data_ptr(), len(row) - 1, src, 4096))
                    kinds.append(("bfs", (d, want)))
                else:
                    roots.append(gt.treesum_root(*[t.data_ptr() for t in tree], 1 << 17, 0, 32))
                    kinds.append(("v", tree_sum))
            first = gt.serve_enqueue(roots)
            for k, kind in enumerate(kinds):
                expect[first + k] = kind
        poll_all(set(expect))
        slots = sorted(expect)
        for s, r in zip(slots, gt.serve_results(slots)):
            kind, want = expect[s]
            assert r.status == gt.ROOT_DONE
            if kind == "v":
                assert r.value == want
            else:
                d, ref = want
                assert np.array_equal(d.cpu().numpy(), ref)
        st = gt.serve_shutdown()
        assert st.status == 0
        assert st.as_dict()["overflow_pushes"] > 0
    finally:
        gt.gtap_finalize()


def test_serve_ring_refuses_more_than_it_holds():
    gt.gtap_initialize(gt.default_config())
    try:
        gt.serve_start(ring_capacity=8)
        first = gt.serve_enqueue([gt.fib_root(10)] * 8)
        assert first == 0
        with pytest.raises(gt.GtapError) as e:
            gt.serve_enqueue([gt.fib_root(10)])   # 8 roots not yet polled: no free slot
        assert e.value.code == 3
        poll_all(set(range(8)))
        res = gt.serve_results(list(range(8)))
        assert all(r.value == 55 for r in res)
        # slots are free again once polled; a reused slot starts from zero
        # (n-queens adds its solutions into the root's value)
        first = gt.serve_enqueue([gt.nq_root(6)] * 4)
        assert first == 8
        poll_all(set(range(4)))
        res = gt.serve_results(list(range(4)))
        assert all(r.value == 4 and r.tasks == orc.nq_tasks(6, 5) for r in res)
        gt.serve_shutdown()
        # results stay readable after the session ends
        assert all(r.value == 4 for r in gt.serve_results(list(range(4))))
    finally:
        gt.gtap_finalize()


def test_serve_calls_outside_a_session_fail_cleanly():
    gt.gtap_initialize(gt.default_config())
    try:
        with pytest.raises(gt.GtapError):
            gt.serve_enqueue([gt.fib_root(5)])
        with pytest.raises(gt.GtapError):
            gt.serve_shutdown()
        # a batch launch while serving is refused
        gt.serve_start(ring_capacity=16)
        with pytest.raises(gt.GtapError):
            gt.launch([gt.fib_root(5)])
        gt.serve_shutdown()
        res, st = gt.launch([gt.fib_root(12)])
        assert res[0].value == 144
    finally:
        gt.gtap_finalize()
