"""Failure detection on the GPU without a GPU fault (B200 only).

Each case drives a deterministic, bounded failure (exhausted id pool, full
spawn buffer, watchdog, unknown task kind): the kernel records the first
error, raises its abort flag and every worker returns; the host reads the
status, the context stays usable, and the next launch is correct.
"""
import ctypes

import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu


def launch_rc(root):
    arr = (gt.Root * 1)(root)
    res = (gt.RootResult * 1)()
    return gt.lib().gtap_launch(arr, 1, res, None, None)


def healthy_afterwards():
    gt.gtap_initialize(gt.default_config())
    try:
        res, st = gt.launch([gt.fib_root(22)])
        assert res[0].value == orc.fib(22)
        assert gt.gtap_get_runtime_error_code() == 0
    finally:
        gt.gtap_finalize()


def test_id_pool_exhausted_reports_and_recovers():
    # one warp running n-queens(12) keeps hundreds of ready tasks per row
    # level (32 lanes x ~8 children): far more than the 128 ids of this arena
    gt.gtap_initialize(gt.default_config(grid=1, block=32, total_ids=128, ids_per_worker=64))
    try:
        rc = launch_rc(gt.nq_root(12))
        assert rc == 6, rc     # TASK_ID_POOL_LOW_HEADROOM / exhausted
        rep = gt.gtap_get_error_report()
        assert rep["valid"] == 1 and rep["code"] == 6
    finally:
        gt.gtap_finalize()
    healthy_afterwards()


def test_spawn_buffer_overflow_reports():
    # cilksort tasks spawn 4 children each that their parent waits for: 32 lanes
    # stage 128 per round, twice this staging capacity.  (Children nobody waits
    # for, as in n-queens, spill to the overflow queue instead of failing.)
    import torch
    gt.gtap_initialize(gt.default_config(spawn_capacity=64))
    try:
        n = 1 << 16
        src = torch.arange(n, 0, -1, dtype=torch.int32, device="cuda")
        arr = torch.empty_like(src)
        tmp = torch.empty_like(src)
        rc = launch_rc(gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n))
        assert rc == 7, rc
        res, st = gt.launch([gt.nq_root(12)])    # detached children: spill, still correct
        assert res[0].value == 14200
    finally:
        gt.gtap_finalize()
    healthy_afterwards()


def test_watchdog_timeout_returns():
    gt.gtap_initialize(gt.default_config(watchdog_ms=1))
    try:
        rc = launch_rc(gt.fib_root(38))
        assert rc == gt.ERROR_TIMEOUT, rc
    finally:
        gt.gtap_finalize()
    healthy_afterwards()


def test_unknown_kind_rejected_on_device():
    gt.gtap_initialize(gt.default_config())
    try:
        rc = launch_rc(gt.Root(kind=99))
        assert rc == 10, rc
        # same runtime, next launch is clean
        res, st = gt.launch([gt.fib_root(15)])
        assert res[0].value == 610
    finally:
        gt.gtap_finalize()


@pytest.mark.parametrize("root", [gt.fib_root(65), gt.nq_root(33), gt.nq_root(8, 256)])
def test_out_of_range_root_rejected_on_device(root):
    # fib's serial leaf handles n <= 64; n-queens has at most 32 columns and
    # packs its cutoff into 8 bits
    gt.gtap_initialize(gt.default_config())
    try:
        rc = launch_rc(root)
        assert rc == 11, rc   # GTAP_ERROR_INVALID_ARGUMENT
        res, st = gt.launch([gt.fib_root(15)])
        assert res[0].value == 610
    finally:
        gt.gtap_finalize()
