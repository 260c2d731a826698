"""The lowered pragma programs (tests/pragma) run on the CPU under the
task-ABI emulator of tests/emu (thread mode), in three task orders, for both
result schemes of gtap_b200.lower: retained child frames (the default) and
--results parent.  Their results must equal the oracle's, as the GPU tests
require of the same programs on the B200.  This checks the lowering's state
machines -- resume labels in branches, frame hoisting, result slots, result
delivery into the parent's frame, frame write-back -- apart from the GPU
runtime."""
import json
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from gtap_b200.lower import lower_source
from tests import oracle_lib as orc
from tests.test_gpu_pragma import walk_expect

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRAGMA = os.path.join(ROOT, "tests", "pragma")
EMU = os.path.join(ROOT, "tests", "emu")
CXX = os.environ.get("CXX", "g++")

PROGRAMS = {
    "fib_pragma": "",
    "walk_pragma": "",
    "fib_queues_pragma": "-DGTAP_NUM_QUEUES=3",
    "cilksort_pragma": "",
    "nq_pragma": "-DGTAP_ASSUME_NO_TASKWAIT",
    "bary_tree_pragma": "",
}
ORDERS = [("lifo", 1), ("fifo", 1), ("random", 7)]


@pytest.fixture(scope="module")
def emu_bins(tmp_path_factory):
    if shutil.which(CXX) is None:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("emu")
    bins = {}
    for name, defs in PROGRAMS.items():
        with open(os.path.join(PRAGMA, name + ".cu")) as f:
            src = f.read()
        for results in ("retain", "parent"):
            text = lower_source(src, mode="thread", results=results)
            text = re.sub(r"(\w+)<<<[^>]*>>>\(", r"\1(", text)     # a launch is a call on the host
            cu = d / ("%s_%s.cpp" % (name, results))
            cu.write_text(text)
            exe = d / ("%s_%s" % (name, results))
            cmd = [CXX, "-std=c++17", "-O1", "-w", "-I", EMU, str(cu), "-o", str(exe)] + defs.split()
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
            assert r.returncode == 0, r.stderr[-3000:]
            bins[(name, results)] = str(exe)
    return bins


def run(exe, order, seed, *args):
    env = dict(os.environ, GTAP_EMU_ORDER=order, GTAP_EMU_SEED=str(seed))
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("results", ["retain", "parent"])
@pytest.mark.parametrize("order,seed", ORDERS)
def test_fib(emu_bins, results, order, seed):
    for n, cutoff in [(0, 0), (1, 0), (2, 0), (18, 0), (22, 9)]:
        r = run(emu_bins[("fib_pragma", results)], order, seed, n, cutoff, 2)
        assert r["error_code"] == 0 and r["results"] == [orc.fib(n)] * 2
        r = run(emu_bins[("fib_queues_pragma", results)], order, seed, n, cutoff, 1)
        assert r["error_code"] == 0 and r["results"] == [orc.fib(n)]


@pytest.mark.parametrize("results", ["retain", "parent"])
@pytest.mark.parametrize("order,seed", ORDERS)
def test_walk(emu_bins, results, order, seed):
    for depth, ident in [(0, 5), (1, 0), (1, 1), (1, 2), (6, 0), (9, 1), (10, 2)]:
        r = run(emu_bins[("walk_pragma", results)], order, seed, depth, ident)
        assert r["error_code"] == 0 and r["result"] == walk_expect(depth, ident)


@pytest.mark.parametrize("results", ["retain", "parent"])
@pytest.mark.parametrize("order,seed", ORDERS)
def test_cilksort_and_nq(emu_bins, results, order, seed):
    for n in [1, 63, 1000, 20011]:
        r = run(emu_bins[("cilksort_pragma", results)], order, seed, n, 3)
        assert r["error_code"] == 0 and r["sorted"] is True
    for n, cutoff in [(4, 3), (8, 7), (9, 4)]:
        r = run(emu_bins[("nq_pragma", results)], order, seed, n, cutoff)
        assert r["error_code"] == 0 and r["result"] == orc.nq(n)


@pytest.mark.parametrize("results", ["retain", "parent"])
@pytest.mark.parametrize("order,seed", ORDERS)
def test_bary_tree(emu_bins, results, order, seed):
    for D, B, mem_ops, iters, log2n in [(0, 3, 4, 4, 8), (5, 3, 8, 16, 10), (8, 4, 16, 32, 12)]:
        s = 3 + D
        r = run(emu_bins[("bary_tree_pragma", results)], order, seed, D, B, mem_ops, iters, log2n, s, 1)
        assert r["error_code"] == 0
        assert (r["sum"], r["nodes"]) == orc.bary_tree(D, B, mem_ops, iters, orc.bary_input(s, 1 << log2n))


def test_emulator_catches_a_broken_lowering(emu_bins, tmp_path):
    """A planted mistake -- the retained child's id released before its result
    is read -- must show up: the freed frame is poisoned."""
    with open(os.path.join(PRAGMA, "fib_pragma.cu")) as f:
        text = lower_source(f.read(), mode="thread")
    good = ("        a = ((__gtap_frame_fib*)__gtap_get_task_data(__f->__child0))->__ret;\n"
            "        b = ((__gtap_frame_fib*)__gtap_get_task_data(__f->__child1))->__ret;\n"
            "        __gtap_release_task_id(__f->__child0);\n")
    assert good in text
    bad = ("        __gtap_release_task_id(__f->__child0);\n"
           "        a = ((__gtap_frame_fib*)__gtap_get_task_data(__f->__child0))->__ret;\n"
           "        b = ((__gtap_frame_fib*)__gtap_get_task_data(__f->__child1))->__ret;\n")
    text = re.sub(r"(\w+)<<<[^>]*>>>\(", r"\1(", text.replace(good, bad))
    cu = tmp_path / "broken.cpp"
    cu.write_text(text)
    exe = tmp_path / "broken"
    r = subprocess.run([CXX, "-std=c++17", "-O1", "-w", "-I", EMU, str(cu), "-o", str(exe)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = run(str(exe), "lifo", 1, 10, 0, 1)
    assert out["results"] != [orc.fib(10)]


def test_emulator_catches_a_missing_write_back(emu_bins, tmp_path):
    """--results parent: without the write-back before a join, the locals a
    task set before suspending are lost when it resumes from its frame."""
    with open(os.path.join(PRAGMA, "walk_pragma.cu")) as f:
        text = lower_source(f.read(), mode="thread", results="parent")
    assert text.count("*__fm = *__f; ") == 3
    text = re.sub(r"(\w+)<<<[^>]*>>>\(", r"\1(", text.replace("*__fm = *__f; ", ""))
    cu = tmp_path / "no_write_back.cpp"
    cu.write_text(text)
    exe = tmp_path / "no_write_back"
    r = subprocess.run([CXX, "-std=c++17", "-O1", "-w", "-I", EMU, str(cu), "-o", str(exe)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = run(str(exe), "lifo", 1, 6, 0)
    assert out["result"] != walk_expect(6, 0)


@pytest.mark.parametrize("order,seed", ORDERS)
def test_hand_lowered_programs(tmp_path, order, seed):
    """The hand-lowered reference programs (tests/lowered) follow the same
    protocol under the emulator (the cilksort one holds inline PTX loads and
    runs on the GPU only)."""
    if shutil.which(CXX) is None:
        pytest.skip("no host C++ compiler")
    for name, defs, args, check in [
        ("fib_lowered", "", (22, 0, 1), lambda r: r["result"] == orc.fib(22)),
        ("fib_lowered", "", (24, 10, 1), lambda r: r["result"] == orc.fib(24)),
        ("nq_lowered", "-DGTAP_ASSUME_NO_TASKWAIT", (9, 4, 1), lambda r: r["result"] == orc.nq(9)),
    ]:
        with open(os.path.join(ROOT, "tests", "lowered", name + ".cu")) as f:
            text = re.sub(r"(\w+)<<<[^>]*>>>\(", r"\1(", f.read())
        cu = tmp_path / (name + ".cpp")
        cu.write_text(text)
        exe = tmp_path / name
        r = subprocess.run([CXX, "-std=c++17", "-O1", "-w", "-I", EMU, str(cu), "-o", str(exe)] + defs.split(),
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        out = run(str(exe), order, seed, *args)
        assert out["error_code"] == 0 and check(out), out


EDGE_MAIN = r"""
__device__ int d_result;

__global__ void exec_kernel(int n) {
    #pragma gtap entry
    d_result = f(n);
}

int main(int argc, char** argv) {
    const int n = atoi(argv[1]);
    gtap_initialize();
    exec_kernel<<<GTAP_GRID_SIZE, GTAP_BLOCK_SIZE>>>(n);
    gtap_synchronize();
    int result = -1, code = 0;
    cudaMemcpyFromSymbol(&result, d_result, sizeof(int));
    gtap_get_runtime_error_code(&code);
    printf("{\"result\": %d, \"error_code\": %d}\n", result, code);
    return code != 0;
}
"""


@pytest.mark.parametrize("results", ["retain", "parent"])
@pytest.mark.parametrize("name,expect", [
    ("comments_strings", lambda n: orc.fib(n)),      # fib with comments and strings holding braces
    ("else_if", lambda n: orc.fib(n)),               # fib through an else-if chain, a taskwait per branch
    ("decl_init", lambda n: 0 if n == 0 else 1),     # f(n) = f(n - 1), from a spawn-initialised local
])
def test_edge_programs_run(tmp_path, results, name, expect):
    if shutil.which(CXX) is None:
        pytest.skip("no host C++ compiler")
    from tests.test_lower_cpu import EDGE
    from gtap_b200.lower import LoweringError
    if results == "parent" and name == "decl_init":
        # --results parent wants a plain local or parameter on the left
        with pytest.raises(LoweringError):
            lower_source(EDGE[name] + EDGE_MAIN, mode="thread", results=results)
        return
    text = lower_source(EDGE[name] + EDGE_MAIN, mode="thread", results=results)
    text = re.sub(r"(\w+)<<<[^>]*>>>\(", r"\1(", text)
    cu = tmp_path / (name + ".cpp")
    cu.write_text("#include <cstdlib>\n" + text)
    exe = tmp_path / name
    r = subprocess.run([CXX, "-std=c++17", "-O1", "-w", "-I", EMU, str(cu), "-o", str(exe)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    for order, seed in ORDERS:
        for n in (0, 1, 2, 11):
            out = run(str(exe), order, seed, n)
            assert out["error_code"] == 0 and out["result"] == expect(n), (order, n, out)


def build_block(tmp_path, name, text, defs=""):
    """A block-mode program for the block emulator (tests/emu/gtap_block.cuh):
    launches run on a block of 32 host threads."""
    text = re.sub(r"(\w+)<<<[^>]*>>>\((.*)\);", r"emu_launch([&] { \1(\2); });", text)
    cu = tmp_path / (name + ".cpp")
    cu.write_text(text)
    exe = tmp_path / name
    r = subprocess.run([CXX, "-std=c++17", "-O1", "-w", "-pthread", "-I", EMU, "-DGTAP_BLOCK_SIZE=32", str(cu),
                        "-o", str(exe)] + defs.split(), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(exe)


@pytest.fixture(scope="module")
def block_bins(tmp_path_factory):
    if shutil.which(CXX) is None:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("emu_block")
    bins = {}
    for name in ("tree_block_pragma", "bary_block_pragma"):
        with open(os.path.join(PRAGMA, name + ".cu")) as f:
            bins[name] = build_block(d, name, lower_source(f.read()))
    with open(os.path.join(ROOT, "tests", "lowered", "tree_block_lowered.cu")) as f:
        bins["tree_block_lowered"] = build_block(d, "tree_block_lowered", f.read())
    return bins


@pytest.mark.parametrize("order,seed", ORDERS)
def test_block_mode_programs(block_bins, order, seed):
    from tests.test_gpu_dropin_block import tree_expect
    for height, work in [(0, 10), (3, 100), (7, 300)]:
        r = run(block_bins["tree_block_pragma"], order, seed, height, work)
        assert r["error_code"] == 0 and r["result"] == tree_expect(height, work)
        r = run(block_bins["tree_block_lowered"], order, seed, height, work, 1)
        assert r["error_code"] == 0 and r["result"] == tree_expect(height, work)
    for D, B, mem_ops, iters, log2n in [(0, 3, 4, 4, 8), (5, 3, 64, 256, 10), (8, 4, 40, 70, 12)]:
        s = 5 + D
        r = run(block_bins["bary_block_pragma"], order, seed, D, B, mem_ops, iters, log2n, s, 1)
        assert r["error_code"] == 0 and r["threads"] == 32
        assert (r["sum"], r["nodes"]) == orc.bary_tree_block(D, B, mem_ops, iters, 32, orc.bary_input(s, 1 << log2n))
