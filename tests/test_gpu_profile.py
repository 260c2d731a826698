"""Profile timelines (B200 only): the CSV files gtap_write_profile writes in
the reference's layout (runtime/detail/thread/gtap_profile_thread.cuh:188-268,
runtime/detail/block/gtap_profile_block.cuh), in thread and block mode.

Every execution is inside one "working" span, so the tasks counted over a
worker's spans add up to the executions the run statistics report, as long
as no worker ran out of samples."""
import csv

import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

FILES = ("timeline_having_task", "statistics_having_task", "timeline_working", "statistics_working")


def read(path):
    with open(path) as f:
        return list(csv.DictReader(f))


def check_profile(tmp_path, unit, st, samples):
    gt.gtap_visualize_profile("app", str(tmp_path))
    tables = {name: read(tmp_path / ("app_%s_%s.csv" % (unit, name))) for name in FILES}
    stats = tables["statistics_working"]
    assert len(stats) == st.workers
    assert list(stats[0].keys()) == ["%s_id" % unit, "total_samples", "first_activity_ms", "last_activity_ms",
                                     "duration_ms", "total_tasks"]
    assert max(int(r["total_samples"]) for r in stats) < samples // 2   # no worker ran out of samples
    assert sum(int(r["total_tasks"]) for r in stats) == st.counters[1]   # executions
    working = tables["timeline_working"]
    assert {r["state_description"] for r in working} == {"Working", "NotWorking"}
    having = tables["timeline_having_task"]
    assert any(r["state_description"] == "Having" for r in having)
    for r in stats:
        assert float(r["duration_ms"]) >= 0.0


def test_thread_mode_profile(tmp_path):
    import torch
    torch.cuda.init()
    gt.gtap_initialize(gt.default_config(profile_samples=512))
    try:
        res, st = gt.launch([gt.fib_root(20), gt.nq_root(8)])
        assert res[0].value == orc.fib(20) and res[1].value == orc.nq(8)
        check_profile(tmp_path, "warp", st, 512)
    finally:
        gt.gtap_finalize()


def test_block_mode_profile(tmp_path):
    import torch
    torch.cuda.init()
    gt.gtap_initialize(gt.default_config(mode=gt.MODE_BLOCK, profile_samples=512))
    try:
        n = 1 << 18
        keys = orc.keys(3, n)
        src = torch.from_numpy(keys).cuda()
        arr = torch.empty_like(src)
        tmp = torch.empty_like(src)
        res, st = gt.launch([gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 2048, 2048)])
        assert np.array_equal(arr.cpu().numpy(), np.sort(keys))
        check_profile(tmp_path, "block", st, 512)
    finally:
        gt.gtap_finalize()
