"""The bench's full-size configurations, each checked against the oracle on
the B200 (not only inside bench.py):

- block-mode cilksort of 2^26 std::mt19937(42) keys, cutoffs 2048/2048: the
  sorted output byte-identical to the oracle's cilksort recursion (which is a
  plain sort of the same keys), and its task count;
- thread-mode mergesort of 2^24 keys, cutoff 128 (parallel merges above 256
  keys): sorted output equal to a plain sort of the same keys;
- thread-mode cilksort of 10^8 keys, the reference's largest published
  configuration (evaluation/2-comparison/cilksort/cilksort_performance_results.csv:11):
  sorted output equal to a plain sort of the same keys;
- n-queens(13) with cutoff 7 (evaluation/2-comparison/nq/nq_performance_results.csv:14):
  73712 solutions and the oracle's task count;
- the 4096-root mix through the host-buffer entry point (copies overlapped
  with three launches): every result and every sorted byte equal to the
  device-resident launch of the same roots, which tests/test_gpu_mix.py checks
  against the oracle.
"""
import os

import numpy as np
import pytest

import gtap_b200 as gt
from gtap_b200.autotune import load_tuned
from gtap_b200.workloads import MERGE_CUTOFF, SORT_CUTOFF, Mix
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sort_run(mode, make_root, n, seed=42, oracle_tasks=None, **cfg):
    import torch
    torch.cuda.init()
    keys = orc.keys(seed, n)
    src = torch.from_numpy(keys).cuda()
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    gt.gtap_initialize(gt.default_config(mode=mode, **cfg))
    try:
        res, st = gt.launch([make_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n)])
    finally:
        gt.gtap_finalize()
    assert st.status == 0 and res[0].status == gt.ROOT_DONE
    return keys, arr.cpu().numpy(), res[0]


def test_block_cilksort_2p26():
    n = 1 << 26
    keys, out, r = _sort_run(gt.MODE_BLOCK, lambda s, a, t, n: gt.cilksort_root(s, a, t, n, 2048, 2048), n)
    want, s_tasks, m_tasks = orc.cilksort(keys, 2048, 2048)
    assert np.array_equal(out, want)
    assert r.tasks == s_tasks + m_tasks


def test_thread_mergesort_2p24():
    n = 1 << 24
    keys, out, r = _sort_run(gt.MODE_THREAD, lambda s, a, t, n: gt.mergesort_root(s, a, t, n, 128, 256), n)
    assert np.array_equal(out, np.sort(keys))


def test_thread_cilksort_1e8():
    n = 100_000_000
    keys, out, r = _sort_run(gt.MODE_THREAD, lambda s, a, t, n: gt.cilksort_root(s, a, t, n, 64, 256), n)
    assert np.array_equal(out, np.sort(keys))


def test_nq13_cutoff7():
    gt.gtap_initialize(gt.default_config())
    try:
        res, st = gt.launch([gt.nq_root(13, 7)])
    finally:
        gt.gtap_finalize()
    assert res[0].value == 73712 == orc.nq(13)
    assert res[0].tasks == orc.nq_tasks(13, 7)


def test_mix_4096_through_host_buffers():
    import torch
    torch.cuda.init()
    mix = Mix(gt, 4096)
    src, arr, tmp = mix.device_slabs()
    droots = mix.roots(gt, src.data_ptr(), arr.data_ptr(), tmp.data_ptr())
    pin_src = torch.from_numpy(mix.keys).pin_memory()
    pin_out = torch.zeros_like(pin_src).pin_memory()
    hroots = mix.roots(gt, pin_src.data_ptr(), pin_out.data_ptr(), 0)
    for r in hroots:   # the host-buffer entry point allocates the scratch itself
        if r.kind == gt.KIND_CILKSORT:
            r.p2 = None
    gt.gtap_initialize(gt.default_config(**load_tuned(os.path.join(ROOT, "gtap_b200", "tuned", "b200_mix.json"))))
    try:
        dres, dst = gt.launch(droots)
        hres, hst, hin, hout = gt.run_host(hroots)
    finally:
        gt.gtap_finalize()
    assert dst.status == 0 and hst.status == 0 and hst.launches == 3
    assert [(r.value, r.tasks, r.status, r.index) for r in hres] == [(r.value, r.tasks, r.status, r.index) for r in dres]
    assert np.array_equal(pin_out.numpy(), arr.cpu().numpy())
    assert hin == 4 * mix.total_keys + 56 * 4096 and hout == 4 * mix.total_keys + 40 * 4096
