"""Drop-in task ABI (include/gtap_thread.cuh) on the GPU (B200 only).

Programs hand-lowered to the reference's task ABI (tests/lowered/*.cu: the
switch state machines clang-gtap emits for `#pragma gtap task / taskwait /
entry`) are compiled against this repository's gtap_thread.cuh and run as
ordinary executables: gtap_initialize(), exec_kernel<<<GRID, BLOCK>>>,
gtap_synchronize(), gtap_reset() between repetitions, gtap_finalize().  Their
results must equal the oracle's.

With GTAP_RUN_REFERENCE_GPU=1, and when the reference runtime was built from
the reference sources (oracle/Makefile ref-gpu -> oracle/_ref/), the same
lowered fib also runs on the reference runtime and both times are printed.
That comparison is opt-in: the reference runtime traps after recording an
error (its n-queens build stopped with "task id pool exhausted" here, and
its per-warp id rings can wrap on other inputs), so the default GPU suite
never runs reference GPU code.
"""
import json
import os
import statistics
import subprocess

import pytest

from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "lowered", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


@pytest.fixture(scope="module")
def bins():
    from gtap_b200.build import build_lowered
    return {os.path.basename(p): p for p in build_lowered()}


def run(exe, *args, timeout=180):
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("name", ["fib_ref_geometry", "fib_b200"])
@pytest.mark.parametrize("n,cutoff", [(0, 0), (1, 0), (2, 0), (20, 0), (27, 0), (30, 12), (32, 20)])
def test_fib_lowered_dropin(bins, name, n, cutoff):
    r = run(bins[name], n, cutoff, 2)
    assert r["error_code"] == 0
    assert r["result"] == orc.fib(n)


def test_fib_lowered_relaunch_after_reset(bins):
    # five launches in one process, gtap_reset() between them
    r = run(bins["fib_b200"], 25, 0, 5)
    assert r["result"] == orc.fib(25) and len(r["ms"]) == 5


def _median(r):
    return statistics.median(r["ms"][1:] if len(r["ms"]) > 1 else r["ms"])


REFERENCE_GPU = os.environ.get("GTAP_RUN_REFERENCE_GPU") == "1"


@pytest.mark.skipif(not REFERENCE_GPU, reason="set GTAP_RUN_REFERENCE_GPU=1 to run the reference GPU build")
@pytest.mark.parametrize("n,cutoff,ref_exe", [(30, 0, "fib_ref"), (34, 12, "fib_ref_c12")])
def test_fib_same_results_as_reference_build(bins, n, cutoff, ref_exe):
    exe = os.path.join(REF, ref_exe)
    if not os.path.exists(exe):
        pytest.skip("%s not built" % ref_exe)
    ref = run(exe, n, cutoff, 6)
    ours = [run(bins[name], n, cutoff, 6) for name in ("fib_ref_geometry", "fib_b200")]
    assert ref["result"] == orc.fib(n)
    for o in ours:
        assert o["result"] == ref["result"]
    print("\nfib(%d) cutoff %d: reference build %.4f ms; drop-in (reference geometry) %.4f ms; drop-in (B200 "
          "geometry) %.4f ms" % (n, cutoff, _median(ref), _median(ours[0]), _median(ours[1])))


@pytest.mark.parametrize("name", ["nq_ref_geometry", "nq_b200"])
@pytest.mark.parametrize("n,cutoff", [(1, 0), (4, 3), (8, 7), (10, 3), (12, 5)])
def test_nq_lowered_dropin(bins, name, n, cutoff):
    r = run(bins[name], n, cutoff, 2)
    assert r["error_code"] == 0
    assert r["result"] == orc.nq(n)


@pytest.mark.parametrize("name", ["cilksort_ref_geometry", "cilksort_b200"])
@pytest.mark.parametrize("n", [1, 63, 64, 1000, 100003, 1 << 20])
def test_cilksort_lowered_dropin(bins, name, n):
    r = run(bins[name], n, 2)
    assert r["error_code"] == 0
    assert r["sorted"] is True
