"""Exactly-once behaviour of the scheduler's queues on the device (B200 only).

gtap_selftest_queues drives every warp through the scheduler's own publish /
pop / steal / overflow-queue code with unique tokens and counts each token
consumed.  Small deques force the split publication (deque + overflow queue)
and full-deque steals, the conditions under which a steal that claims a batch
before its slot reads complete would duplicate tokens.
"""
import pytest

import gtap_b200 as gt

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg", [dict(deque_capacity=64), dict(deque_capacity=64, steal_batch=1),
                                 dict(deque_capacity=128, block=1024), dict(deque_capacity=4096)])
@pytest.mark.parametrize("rounds,per_round,mode", [(20, 100, 2), (20, 100, 7), (60, 32, 7), (150, 12, 3)])
def test_queues_exactly_once(cfg, rounds, per_round, mode):
    gt.gtap_initialize(gt.default_config(total_ids=1 << 24, **cfg))
    try:
        rc, d = gt.selftest_queues(rounds, per_round, mode)
        assert rc == 0, d
        assert d["duplicates"] == 0 and d["lost"] == 0
        assert d["produced"] == d["consumed"] > 0
    finally:
        gt.gtap_finalize()
