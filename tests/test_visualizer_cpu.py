"""The reference's profile visualiser on this runtime's profiler CSVs (CPU).

tests/golden/profile/ holds the four CSV files gtap_visualize_profile wrote
for a small fib run on a B200 (tests/golden/make_profile_fixture.py).  The
reference reads them with examples/fib_profile/visualize_profile.py; its
data loading (load_data and _compute_utilization, :72-127) needs only pandas,
its plots need matplotlib, which this image lacks.  So matplotlib is replaced
by inert stand-in modules at import, and the script's own parsing runs on the
committed files.  The column checks below hold without the reference too.
"""
import csv
import importlib.util
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILE = os.path.join(ROOT, "tests", "golden", "profile")
VISUALIZER = os.path.join(os.environ.get("GTAP_REFERENCE", "/root/reference"), "examples", "fib_profile",
                          "visualize_profile.py")

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(PROFILE, "fib_warp_timeline_working.csv")),
                                reason="profile fixture not generated")


def rows(name):
    with open(os.path.join(PROFILE, name)) as f:
        return list(csv.DictReader(f))


def test_fixture_columns_match_the_reference_layout():
    # runtime/detail/thread/gtap_profile_thread.cuh:188-268 writes these columns
    tl = rows("fib_warp_timeline_working.csv")
    assert list(tl[0]) == ["warp_id", "time_index", "timestamp_ns", "relative_time_ms", "state",
                           "state_description", "tasks_in_batch"]
    st = rows("fib_warp_statistics_working.csv")
    assert list(st[0]) == ["warp_id", "total_samples", "first_activity_ms", "last_activity_ms", "duration_ms",
                           "total_tasks"]
    assert {r["state_description"] for r in tl} == {"Working", "NotWorking"}


def _stub_matplotlib():
    """Inert matplotlib modules: attribute access and calls do nothing."""
    class Inert(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith("__"):
                raise AttributeError(name)
            return Inert(name)

        def __call__(self, *a, **k):
            return Inert("call")

    saved = {k: sys.modules.get(k) for k in ("matplotlib", "matplotlib.pyplot", "matplotlib.patches")}
    mpl = Inert("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = Inert("matplotlib.pyplot")
    plt.rcParams = {}
    mpl.pyplot = plt
    mpl.patches = Inert("matplotlib.patches")
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt
    sys.modules["matplotlib.patches"] = mpl.patches
    return saved


@pytest.mark.skipif(not os.path.exists(VISUALIZER), reason="reference visualiser not present")
def test_reference_visualiser_parses_the_csvs():
    saved = _stub_matplotlib()
    try:
        spec = importlib.util.spec_from_file_location("gtap_ref_visualize_profile", VISUALIZER)
        vis = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(vis)
        timeline, stats, strong = vis.load_data(PROFILE, "fib")
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    assert strong == "Working"
    assert len(timeline) == len(rows("fib_warp_timeline_working.csv"))
    # the statistics file has no utilization column, so the script derived
    # one per warp from the timeline
    assert "utilization_percent" in stats.columns
    util = stats["utilization_percent"]
    assert util.notna().all() and (util >= 0).all() and (util <= 100).all()
    assert util.max() > 0
    assert sorted(stats["warp_id"]) == sorted({int(r["warp_id"]) for r in rows("fib_warp_statistics_working.csv")})
