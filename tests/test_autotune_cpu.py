"""Autotuner search logic on the CPU (no GPU): coordinate descent over a
synthetic cost surface, invalid points, and config overrides."""
import json

from gtap_b200 import autotune as at


def test_coordinate_descent_finds_separable_minimum():
    target = {"warps_per_sm": 12, "block": 128, "steal_batch": 8, "deque_capacity": 1024,
              "probe_width": 4, "victim_policy": 1, "num_queues": 2}

    def cost(p):
        return sum(abs(at.SPACE[k].index(p[k]) - at.SPACE[k].index(target[k])) for k in target) + 1.0

    start = {"warps_per_sm": 8, "block": 256, "deque_capacity": 4096, "steal_batch": 32,
             "probe_width": 16, "victim_policy": 2, "num_queues": 1}
    best, t, trials = at.coordinate_descent(cost, start)
    assert best == target and t == 1.0
    assert len(trials) <= 2 * sum(len(v) for v in at.SPACE.values())


def test_invalid_points_are_skipped():
    start = {"warps_per_sm": 8, "block": 256, "deque_capacity": 4096, "steal_batch": 32,
             "probe_width": 16, "victim_policy": 2, "num_queues": 1}

    def cost(p):
        if p["block"] == 1024:
            return None            # e.g. the runtime refused the configuration
        return 1.0 / p["warps_per_sm"] + (0.5 if p["block"] != 512 else 0.0)

    best, t, _ = at.coordinate_descent(cost, start)
    assert best["block"] == 512 and best["warps_per_sm"] == 32


def test_overrides_and_tuned_file(tmp_path):
    o = at.to_overrides({"warps_per_sm": 16, "block": 128, "steal_batch": 8}, 148)
    assert o == {"block": 128, "steal_batch": 8, "grid": 16 * 148 // 4}
    f = tmp_path / "t.json"
    f.write_text(json.dumps({"best_overrides": o}))
    assert at.load_tuned(str(f)) == o
    assert at.load_tuned(str(tmp_path / "missing.json")) == {}


def test_descent_follows_a_custom_space_and_order():
    """Workloads that search a subset of the axes (block-mode cilksort, mergesort)
    pass their own space and order; axes outside the order keep the start value."""
    space = dict(at.SPACE, warps_per_sm=[16, 32, 48, 64])
    order = ["warps_per_sm", "block"]
    start = {"warps_per_sm": 64, "block": 256, "probe_width": 16}

    def cost(p):
        return abs(p["warps_per_sm"] - 48) + abs(p["block"] - 128) / 64.0 + (p["probe_width"] != 16) * 100

    best, t, trials = at.coordinate_descent(cost, start, space=space, order=order)
    assert best == {"warps_per_sm": 48, "block": 128, "probe_width": 16}
    assert all(tr["point"]["probe_width"] == 16 for tr in trials)


def test_new_axes_are_searched():
    for axis, values in (("join_walk", [0, 2, 4, 8, 32]), ("sub_rounds", [0, 1, 2, 4, 8])):
        assert at.SPACE[axis] == values and axis in at.ORDER


def test_profile_case_closed_form_matches_oracle():
    from gtap_b200.profile_case import fib_value_and_tasks
    from tests import oracle_lib as orc
    for n in (0, 1, 2, 10, 30):
        assert fib_value_and_tasks(n) == (orc.fib(n), orc.fib_tasks(n, 0))
