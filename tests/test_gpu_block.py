"""Block-cooperative mode against the oracle (B200 only).

One task = one CUDA block (reference runtime/detail/block/gtap_runtime_block.cuh).
The spawn trees are the reference recursions, so task counts must equal the
oracle's; sorted outputs must equal a plain sort of the input, BFS depths the
oracle's BFS, sums and counts the oracle's values.
"""
import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

INF = 0x3f3f3f3f


@pytest.fixture(scope="module")
def blk():
    import torch
    torch.cuda.init()
    gt.gtap_initialize(gt.default_config(mode=gt.MODE_BLOCK))
    yield gt
    gt.gtap_finalize()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run1(root):
    res, st = gt.launch([root])
    assert st.status == 0
    return res[0], st


def sort_case(keys, sc, mc):
    import torch
    src = dev(keys)
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    r, st = run1(gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), len(keys), sc, mc))
    assert r.status == gt.ROOT_DONE
    assert np.array_equal(arr.cpu().numpy(), np.sort(keys))
    assert np.array_equal(src.cpu().numpy(), keys)   # the input is left as it was
    _, sort_tasks, merge_tasks = orc.cilksort(keys, sc, mc)
    assert r.tasks == sort_tasks + merge_tasks
    return r, st


@pytest.mark.parametrize("n", [1, 2, 63, 1000, 2047, 2048, 4095, 4096, 100003, 1 << 20])
def test_cilksort_cutoffs_2048(blk, n):
    sort_case(orc.keys(n, n), 2048, 2048)


@pytest.mark.parametrize("n,sc,mc", [(50000, 64, 256), (77777, 2049, 2049), (1 << 16, 2, 3), (9999, 513, 2000)])
def test_cilksort_other_cutoffs(blk, n, sc, mc):
    sort_case(orc.keys(3 * n + 1, n), sc, mc)


def test_cilksort_duplicate_heavy_keys(blk):
    rng = np.random.default_rng(5)
    keys = rng.integers(-3, 4, size=(1 << 18) + 7).astype(np.int32)
    keys[::97] = np.iinfo(np.int32).max
    keys[::89] = np.iinfo(np.int32).min
    sort_case(keys, 2048, 2048)


@pytest.mark.parametrize("n,cutoff", [(1, 128), (1000, 128), (1 << 16, 2048), (77777, 2048)])
def test_mergesort(blk, n, cutoff):
    import torch
    keys = orc.keys(11 + n, n)
    src = dev(keys)
    out = torch.empty_like(src)
    tmp = torch.empty_like(src)
    r, st = run1(gt.mergesort_root(src.data_ptr(), out.data_ptr(), tmp.data_ptr(), n, cutoff, 2048))
    assert r.status == gt.ROOT_DONE
    assert np.array_equal(out.cpu().numpy(), np.sort(keys))


@pytest.mark.parametrize("n,cutoff", [(0, 0), (1, 0), (2, 0), (15, 0), (22, 12)])
def test_fib(blk, n, cutoff):
    r, st = run1(gt.fib_root(n, cutoff=cutoff))
    assert r.value == orc.fib(n)
    assert r.tasks == orc.fib_tasks(n, cutoff)


@pytest.mark.parametrize("n", [1, 4, 6, 8])
def test_nq(blk, n):
    r, st = run1(gt.nq_root(n))
    assert r.value == orc.nq(n)
    assert r.tasks == orc.nq_tasks(n, n - 1)


@pytest.mark.parametrize("scale", [8, 12, 15])
def test_bfs(blk, scale):
    import torch
    row, col = gt.gen_rmat(scale, 16, 42 + scale)
    src = gt.max_degree_vertex(row)
    drow, dcol = dev(row), dev(col)
    depth = torch.full((len(row) - 1,), INF, dtype=torch.int32, device="cuda")
    r, st = run1(gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), depth.data_ptr(), len(row) - 1, src))
    assert np.array_equal(depth.cpu().numpy(), orc.bfs(row, col, src))


@pytest.mark.parametrize("n,cutoff", [(1, 32), (1000, 1), (1 << 16, 64)])
def test_treesum(blk, n, cutoff):
    left, right, value, size = gt.gen_tree(n, 5)
    d = [dev(x) for x in (left, right, value, size)]
    r, st = run1(gt.treesum_root(*[x.data_ptr() for x in d], n, 0, cutoff))
    assert r.value == orc.tree_sum(left, right, value, 0)


def test_mixed_roots_in_one_launch(blk):
    import torch
    roots, checks, keep = [], [], []
    for i, n in enumerate((3000, 1 << 17, 70001)):
        keys = orc.keys(100 + i, n)
        src = dev(keys)
        arr = torch.empty_like(src)
        tmp = torch.empty_like(src)
        keep += [src, arr, tmp]
        roots.append(gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 2048, 2048))
        checks.append(("sort", arr, np.sort(keys)))
    for n in (10, 17):
        roots.append(gt.fib_root(n))
        checks.append(("v", None, orc.fib(n)))
    roots.append(gt.nq_root(7))
    checks.append(("v", None, orc.nq(7)))
    res, st = gt.launch(roots)
    assert st.status == 0
    for r, (kind, buf, want) in zip(res, checks):
        assert r.status == gt.ROOT_DONE
        if kind == "sort":
            assert np.array_equal(buf.cpu().numpy(), want)
        else:
            assert r.value == want
    assert st.counters[0] == sum(r.tasks for r in res)


@pytest.mark.parametrize("sc,mc", [(1, 2048), (2048, 2)])
def test_cutoffs_that_never_end_are_rejected(blk, sc, mc):
    import torch
    src = dev(orc.keys(2, 1000))
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    with pytest.raises(gt.GtapError) as e:
        gt.launch([gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), 1000, sc, mc)])
    assert e.value.code == gt.ERROR_INVALID_ARGUMENT


def test_leaf_cutoff_above_shared_memory_is_rejected(blk):
    # a leaf of more than 2048 keys does not fit the block's staging buffers
    import torch
    src = dev(orc.keys(1, 10000))
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    with pytest.raises(gt.GtapError) as e:
        gt.launch([gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), 10000, 8192, 2048)])
    assert e.value.code == gt.ERROR_INVALID_ARGUMENT
    # the runtime stays usable
    r, st = run1(gt.fib_root(12))
    assert r.value == 144


def test_serve_in_block_mode(blk):
    import time
    gt.serve_start(ring_capacity=32)
    try:
        first = gt.serve_enqueue([gt.fib_root(n) for n in range(5, 15)] + [gt.nq_root(6)])
        pending = set(range(first, first + 11))
        t0 = time.time()
        while pending and time.time() - t0 < 20:
            for i in gt.serve_poll(64):
                pending.discard(i)
        assert not pending
        res = gt.serve_results(list(range(first, first + 11)))
        assert [r.value for r in res] == [orc.fib(n) for n in range(5, 15)] + [orc.nq(6)]
    finally:
        st = gt.serve_shutdown()
    assert st.status == 0
