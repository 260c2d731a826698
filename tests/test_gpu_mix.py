"""The benchmark's workload, whole (B200 only): the seeded 4096-root mix in one
persistent launch, with the autotuned configuration the benchmark uses.

Every root is checked against the oracle: fib and n-queens values and task
counts, and for each of the ~1,365 cilksort roots the sorted output byte-for-
byte and the task count (sort plus merge tasks) of the oracle's cilksort
recursion on the same keys (examples/cilksort/cilksort.cu:225-258 compares
the sorted output with std::sort exactly).  A second launch of the same roots
must give the same results.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import gtap_b200 as gt
from gtap_b200.autotune import load_tuned
from gtap_b200.workloads import MERGE_CUTOFF, SORT_CUTOFF, Mix
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_mix_4096_roots_exact():
    import torch
    torch.cuda.init()
    mix = Mix(gt, 4096)
    # the same mix as the oracle's generators
    kind, param, seed = orc.root_mix(42, 4096)
    assert np.array_equal(kind, mix.kind) and np.array_equal(param, mix.param) and np.array_equal(seed, mix.seed)
    src, arr, tmp = mix.device_slabs()
    roots = mix.roots(gt, src.data_ptr(), arr.data_ptr(), tmp.data_ptr())
    gt.gtap_initialize(gt.default_config(**load_tuned(os.path.join(ROOT, "gtap_b200", "tuned", "b200_mix.json"))))
    try:
        res, st = gt.launch(roots)
        out = arr.cpu().numpy()
        res2, _ = gt.launch(roots)
        out2 = arr.cpu().numpy()
    finally:
        gt.gtap_finalize()
    assert st.status == 0
    assert sum(r.tasks for r in res) == st.counters[0]

    sorts = np.nonzero(mix.kind == 2)[0]

    def oracle_sort(i):
        o, n = int(mix.offsets[i]), int(mix.param[i])
        want, s_tasks, m_tasks = orc.cilksort(mix.keys[o:o + n], SORT_CUTOFF, MERGE_CUTOFF)
        return i, want, s_tasks + m_tasks

    with ThreadPoolExecutor(os.cpu_count() or 4) as pool:
        oracle = {i: (want, t) for i, want, t in pool.map(oracle_sort, sorts)}

    bad = []
    for i, r in enumerate(res):
        k, p = int(mix.kind[i]), int(mix.param[i])
        if r.status != gt.ROOT_DONE:
            bad.append((i, "status", r.status))
            continue
        if k == 0:
            if (r.value, r.tasks) != (orc.fib(p), orc.fib_tasks(p, 0)):
                bad.append((i, "fib", p, r.value, r.tasks))
        elif k == 1:
            if (r.value, r.tasks) != (orc.nq(p), orc.nq_tasks(p, p - 1)):
                bad.append((i, "nq", p, r.value, r.tasks))
        else:
            o = int(mix.offsets[i])
            want, tasks = oracle[i]
            if not np.array_equal(out[o:o + p], want):
                bad.append((i, "cilksort output", p))
            if r.tasks != tasks:
                bad.append((i, "cilksort tasks", p, r.tasks, tasks))
    assert not bad, bad[:10]
    assert len(sorts) > 1000 and mix.total_keys > 1 << 27
    # the repeated launch: same values, same task counts, same sorted bytes
    assert [(r.value, r.tasks, r.status) for r in res2] == [(r.value, r.tasks, r.status) for r in res]
    assert np.array_equal(out2, out)
