"""bench.py's host logic on CPU: the clock-sample summary that decides
whether a run is kept (median SM clock, throttle reasons seen under load),
and the algorithmic byte models behind the roofline figures."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


bench = load_bench()

NOT_ACTIVE = "Not Active, Not Active, Not Active, Not Active"


def test_clock_summary_of_a_clean_run():
    lines = ["1965, 1965, 612.4, " + NOT_ACTIVE, "1965, 1965, 640.1, " + NOT_ACTIVE, "1950, 1965, 655.0, " + NOT_ACTIVE]
    c = bench.Clocks.summarize(lines)
    assert c == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}


def test_clock_summary_reports_every_reason_seen():
    lines = ["1965, 1965, 900.0, " + NOT_ACTIVE,
             "1305, 1965, 1000.0, Not Active, Not Active, Not Active, Active",
             "1290, 1965, 1000.0, Active, Not Active, Not Active, Active"]
    c = bench.Clocks.summarize(lines)
    assert c["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert c["sm_mhz"] == 1305.0 and c["samples"] == 3


def test_clock_summary_skips_malformed_lines():
    lines = ["", "[N/A], 1965, 600, " + NOT_ACTIVE, "1965, 1965", "1965, 1965, 600.0, " + NOT_ACTIVE]
    c = bench.Clocks.summarize(lines)
    assert c["samples"] == 1 and c["sm_mhz"] == 1965.0
    assert bench.Clocks.summarize([]) == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_cilksort_bytes_model():
    assert bench.cilksort_bytes(1000, 2048) == 8 * 1000                   # one leaf (n < cutoff): read + write
    assert bench.cilksort_bytes(60, 16) == 16 * 60 + 8 * 60               # one inner node over four 15-key leaves
    assert bench.cilksort_bytes(64, 16) == 16 * 64 + 4 * (16 * 16 + 8 * 16)   # 16-key quarters split once more
    assert bench.cilksort_bytes(1 << 26, 2048) == 9126805504              # the 2^26-key workload's figure


def test_mergesort_bytes_model():
    assert bench.mergesort_bytes(100, 128) == 800
    assert bench.mergesort_bytes(256, 128) == 8 * 256 * 2                 # one merge over two leaves
    assert bench.mergesort_bytes(1 << 24, 128) == 2415919104              # the 2^24-key workload's figure


def test_reference_arm_runs_without_the_product_library():
    """`bench.py --impl reference` builds the mix with the oracle's generators
    and times the oracle's sequential programs: the product library is never
    mapped into its process, and it prints the same `config` object as the
    GPU arm (workload_config of the same mix built by the library)."""
    import json
    import subprocess
    import sys
    code = ("import sys, json, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', "
            "'--warmup', '1', '--roots', '96', '--cpu-sample-s', '0.2']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'lib_mapped': 'libgtap_b200' in maps, 'oracle_mapped': 'liboracle' in maps}))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [json.loads(ln) for ln in out.stdout.strip().splitlines()]
    line, maps = lines[0], lines[-1]
    assert maps == {"lib_mapped": False, "oracle_mapped": True}
    assert line["impl"] == "reference" and line["unit"] == "tasks/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
    import gtap_b200 as gt
    from gtap_b200.workloads import Mix
    assert line["config"] == bench.workload_config(Mix(gt, 96))


def test_worker_kernels_of_a_split_and_an_unsplit_step():
    split = bench.worker_kernels(100e6, 200e6, 50.0, 25.0, 6000.0)
    assert [k["kernel"] for k in split] == [bench.LIGHT_KERNEL, bench.FULL_KERNEL]
    assert [k["algorithmic_bytes"] for k in split] == [100e6, 200e6]
    assert abs(split[0]["achieved_gbs"] - 2.0) < 1e-9 and abs(split[1]["frac"] - 8.0 / 6000.0) < 1e-12
    one = bench.worker_kernels(100e6, 200e6, 0.0, 75.0, 6000.0)
    assert len(one) == 1 and one[0]["kernel"] == bench.FULL_KERNEL and one[0]["algorithmic_bytes"] == 300e6
    only_light = bench.worker_kernels(100e6, 0, 40.0, 0.0, 6000.0)
    assert [k["kernel"] for k in only_light] == [bench.LIGHT_KERNEL]
