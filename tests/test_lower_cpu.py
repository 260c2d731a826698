"""gtap_b200.lower on CPU: the pragma programs of tests/pragma lower to the
task ABI and the result compiles for sm_100a against the drop-in headers;
programs outside the supported subset are refused with a LoweringError."""
import os
import re
import shutil
import subprocess

import pytest

from gtap_b200.lower import LoweringError, lower_source

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRAGMA = os.path.join(ROOT, "tests", "pragma")
NVCC = os.environ.get("NVCC", "nvcc")


def read(name):
    with open(os.path.join(PRAGMA, name)) as f:
        return f.read()


def test_fib_lowers_to_a_state_machine():
    out = lower_source(read("fib_pragma.cu"))
    assert "#pragma gtap" not in out.replace("#pragma gtap function", "")   # every pragma was consumed
    assert "struct __gtap_frame_fib" in out and "int __ret;" in out
    assert "switch (__gtap_get_task_state(__tid))" in out
    assert "__gtap_set_state_for_join(__tid, __cc, 1, 0)" in out
    assert out.count("__gtap_spawn_task(") == 3           # two in fib, one in the entry task
    assert "__gtap_release_task_id(__f->__child0)" in out
    assert "const size_t __gtap_auto_task_data_size" in out
    assert "__gtap_execute_task_loop_device();" in out
    assert out.startswith("#define GTAP_DIRECT_DISPATCH 1\n")
    assert "if (__fn == (unsigned long long)(void*)&fib__gtap_task) { fib__gtap_task(__frame, __tid, __ctx); return; }" in out
    assert "(void*)&__gtap_entry0)" in out


def test_queue_clauses_reach_the_runtime_calls():
    out = lower_source(read("fib_queues_pragma.cu"))
    assert "fib__gtap_task, (n - 1) & 1, &__f->__child0, true)" in out
    assert "fib__gtap_task, n & 1, &__f->__child1, true)" in out
    assert "__gtap_set_state_for_join(__tid, __cc, 1, 2)" in out


def test_block_mode_follows_the_header():
    out = lower_source(read("tree_block_pragma.cu"))
    assert "__gtap_set_state_for_join_block(__tid, __ctx, 1, 0)" in out
    assert "__syncthreads();" in out                      # child slots cleared before any thread spawns
    assert "if (threadIdx.x == 0) __gtap_release_task_id" in out


def test_result_only_locals_stay_out_of_the_frame():
    out = lower_source(read("fib_pragma.cu"))
    frame = out[out.index("struct __gtap_frame_fib"):]
    frame = frame[:frame.index("};")]
    # a and b only receive the children's results at the one taskwait
    assert frame.split() == ["struct", "__gtap_frame_fib", "{", "int", "n;", "int", "__ret;",
                             "int", "__child0;", "int", "__child1;"]
    body = out[out.index("__device__ void fib__gtap_task(void* __frame, int __tid, TaskContext* __ctx) {"):]
    # both results are read before either id is released
    assert (body.index("b = ((__gtap_frame_fib*)__gtap_get_task_data(__f->__child1))->__ret;")
            < body.index("__gtap_release_task_id(__f->__child0);"))


def test_only_live_locals_go_to_the_frame():
    out = lower_source(read("nq_pragma.cu"))
    frame = out[out.index("struct __gtap_frame_nq"):]
    frame = frame[:frame.index("};")]
    assert "avail" not in frame                           # no taskwait: nothing crosses one
    out = lower_source(read("cilksort_pragma.cu"))
    frame = out[out.index("struct __gtap_frame_csort"):]
    frame = frame[:frame.index("};")]
    assert "int h;" in frame and "int q1;" in frame       # used after the first taskwait


def test_taskwait_in_a_branch_resumes_inside_it():
    out = lower_source(read("walk_pragma.cu"))
    body = out[out.index("__device__ void walk__gtap_task(void* __frame, int __tid, TaskContext* __ctx) {"):]
    # labels 1 and 2 sit in the two branches, 3 at the top level
    assert body.index("case 1:") < body.index("} else {") < body.index("case 2:") < body.index("case 3:")
    assert "int spare; spare = id & 7;" in body                # in scope at a label, not used after it
    assert "__f->k = id % 3;" in body                          # const local kept in the frame
    assert "__f->a = 0; __f->b = 0; __f->own = id;" in body
    assert "    int id = __f->id;\n" in body                     # parameters never written: read once
    assert "&__f->__child2, true" in body and "nullptr, false" in body
    # a conditional spawn's slot is cleared on entry and checked at its join
    assert "__f->__child2 = -1; " in body and "if (__f->__child2 >= 0) __f->a =" in body
    assert "__f->__child0 = -1" not in body
    out = lower_source(read("tree_block_pragma.cu"))
    assert "int lc = 2 * node + 1;" in out                     # declared in a block that ends before the join


BAD = {
    "taskwait in a loop": """
#pragma gtap function
__device__ void f(int n) {
    for (int i = 0; i < n; ++i) {
        #pragma gtap task
        f(i);
        #pragma gtap taskwait
    }
}
""",
    "taskwait in a switch": """
#pragma gtap function
__device__ void f(int n) {
    switch (n) {
    case 1: {
        #pragma gtap task
        f(n - 1);
        #pragma gtap taskwait
        break;
    }
    default:
        break;
    }
}
""",
    "taskwait without braces": """
#pragma gtap function
__device__ void f(int n) {
    #pragma gtap task
    f(n - 1);
    if (n > 2)
        #pragma gtap taskwait
    return;
}
""",
    "result in a loop": """
#pragma gtap function
__device__ int f(int n) {
    int s = 0;
    for (int i = 0; i < n; ++i) {
        #pragma gtap task
        s = f(i);
    }
    #pragma gtap taskwait
    return s;
}
""",
    "result joined only in a branch": """
#pragma gtap function
__device__ int f(int n) {
    int a = 0;
    #pragma gtap task
    a = f(n - 1);
    if (n > 3) {
        #pragma gtap taskwait
    }
    return a;
}
""",
    "task on a plain function": """
__device__ int g(int n) { return n; }
#pragma gtap function
__device__ void f(int n) {
    #pragma gtap task
    g(n);
}
""",
    "result without a taskwait": """
#pragma gtap function
__device__ int f(int n) {
    int a;
    #pragma gtap task
    a = f(n - 1);
    return a;
}
""",
    "live local declared twice": """
#pragma gtap function
__device__ int f(int n) {
    int a = 0;
    if (n > 1) {
        #pragma gtap task
        a = f(n - 1);
        #pragma gtap taskwait
    } else {
        int a = 1;
        return a;
    }
    return a;
}
""",
    "local shadows a parameter": """
#pragma gtap function
__device__ void f(int n) {
    if (n > 1) {
        int n = 3;
        #pragma gtap task
        f(n - 1);
    }
}
""",
    "class-type local across a taskwait": """
struct P { int x; };
#pragma gtap function
__device__ void f(int n) {
    P p;
    p.x = n;
    #pragma gtap task
    f(n - 1);
    #pragma gtap taskwait
    n = p.x;
}
""",
    "array live across a taskwait": """
#pragma gtap function
__device__ void f(int n) {
    int v[4];
    v[0] = n;
    #pragma gtap task
    f(n - 1);
    #pragma gtap taskwait
    n = v[0];
}
""",
    "no task function": "__device__ int f(int n) { return n; }\n",
    "compound assignment of a result": """
#pragma gtap function
__device__ int f(int n) {
    int a = 0;
    #pragma gtap task
    a += f(n - 1);
    #pragma gtap taskwait
    return a;
}
""",
}


@pytest.mark.parametrize("what", sorted(BAD))
def test_unsupported_programs_are_refused(what):
    with pytest.raises(LoweringError):
        lower_source(BAD[what])


@pytest.mark.skipif(shutil.which(NVCC) is None, reason="nvcc not available")
@pytest.mark.parametrize("src,defs", [
    ("fib_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2"),
    ("nq_pragma.cu", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("cilksort_pragma.cu", "-DGTAP_GRID_SIZE=592 -DGTAP_BLOCK_SIZE=128"),
    ("tree_block_pragma.cu", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128"),
    ("walk_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128"),
    ("fib_queues_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_NUM_QUEUES=3"),
    ("bary_tree_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=8"),
    ("bary_block_pragma.cu", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128"),
])
def test_lowered_program_compiles(tmp_path, src, defs):
    low = tmp_path / ("lowered_" + src)
    low.write_text(lower_source(read(src)))
    cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-diag-suppress", "550",
           "-I", os.path.join(ROOT, "include"), "-c", str(low), "-o", str(tmp_path / "prog.o")] + defs.split()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]


EDGE = {
    # braces and `return` inside comments and string literals stay as written
    "comments_strings": """
#include <stdio.h>
#include "gtap_thread.cuh"
#pragma gtap function
__device__ int f(int n) {
    // a comment with { braces and return 3;
    if (n < 2) { /* } closing brace in a comment */ return n; }
    int a, b;
    #pragma gtap task
    a = f(n - 1);   // trailing comment }
    #pragma gtap task
    b = f(n - 2);
    #pragma gtap taskwait
    if (n == 99) printf("{ return %d; }\\n", a);
    return a + b;
}
""",
    # taskwaits in an else-if chain, a result assigned to the function's own local
    "else_if": """
#include "gtap_thread.cuh"
#pragma gtap function
__device__ int f(int n) {
    int r = 0;
    if (n < 2) {
        return n;
    } else if (n % 2 == 0) {
        int a, b;
        #pragma gtap task
        a = f(n - 1);
        #pragma gtap task
        b = f(n - 2);
        #pragma gtap taskwait
        r = a + b;
    } else {
        int c;
        #pragma gtap task
        c = f(n - 1);
        #pragma gtap task
        r = f(n - 2);
        #pragma gtap taskwait
        r += c;
    }
    return r;
}
""",
    # a declaration initialised by a spawn
    "decl_init": """
#include "gtap_thread.cuh"
#pragma gtap function
__device__ int f(int n) {
    if (n < 2) return n;
    #pragma gtap task
    int a = f(n - 1);
    #pragma gtap taskwait
    return a;
}
""",
}


def test_literals_and_comments_are_kept():
    out = lower_source(EDGE["comments_strings"])
    assert "// a comment with { braces and return 3;" in out
    assert "/* } closing brace in a comment */" in out
    assert 'printf("{ return %d; }\\n", ' in out


def test_else_if_chain_resumes_in_each_branch():
    out = lower_source(EDGE["else_if"])
    body = out[out.index("__device__ void f__gtap_task(void* __frame, int __tid, TaskContext* __ctx) {"):]
    assert body.index("} else if (n % 2 == 0) {") < body.index("case 1:") < body.index("} else {") < body.index("case 2:")


@pytest.mark.skipif(shutil.which(NVCC) is None, reason="nvcc not available")
@pytest.mark.parametrize("name", sorted(EDGE))
def test_edge_programs_compile(tmp_path, name):
    low = tmp_path / (name + ".cu")
    low.write_text(lower_source(EDGE[name]))
    cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-diag-suppress", "550",
           "-I", os.path.join(ROOT, "include"), "-DGTAP_GRID_SIZE=888", "-DGTAP_BLOCK_SIZE=128",
           "-c", str(low), "-o", str(tmp_path / "prog.o")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]


def test_command_line(tmp_path):
    import sys
    out = tmp_path / "fib_lowered.cu"
    r = subprocess.run([sys.executable, "-m", "gtap_b200.lower", os.path.join(PRAGMA, "fib_pragma.cu"), "-o", str(out)],
                       cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert out.read_text() == lower_source(read("fib_pragma.cu"))
    bad = tmp_path / "bad.cu"
    bad.write_text(BAD["taskwait in a loop"])
    r = subprocess.run([sys.executable, "-m", "gtap_b200.lower", str(bad), "-o", str(tmp_path / "x.cu")],
                       cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "line 7: a taskwait inside a loop of 'f' is not supported" in r.stderr
    assert not (tmp_path / "x.cu").exists()
    # --mode overrides the header the program includes
    r = subprocess.run([sys.executable, "-m", "gtap_b200.lower", os.path.join(PRAGMA, "fib_pragma.cu"), "-o",
                        str(out), "--mode", "block"], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "__gtap_set_state_for_join_block" in out.read_text()


# --results parent (thread mode): children write their results into the
# parent's frame; tasks read their frames from the words loaded with the header
def test_parent_results_frame_and_delivery():
    out = lower_source(read("fib_pragma.cu"), results="parent")
    assert out.startswith("#define GTAP_FRAME_WORDS 1\n")
    frame = out[out.index("struct __gtap_frame_fib"):]
    frame = frame[:frame.index("};")]
    assert frame.split() == ["struct", "__gtap_frame_fib", "{", "int", "n;", "int", "a;", "int", "b;",
                             "unsigned", "__dst;"]
    assert "__c->__dst = __gtap_dst(__tid, offsetof(__gtap_frame_fib, a));" in out
    assert "__c->__dst = __gtap_dst(__tid, offsetof(__gtap_frame_fib, b));" in out
    assert "if (__f->__dst) __gtap_deliver<int>(__f->__dst, (__f->a + __f->b));" in out
    assert "*__fm = *__f; if (__gtap_set_state_for_join(__tid, __cc, 1, 0)) return;" in out
    assert "__gtap_release_task_id" not in out and "__child" not in out.split("__gtap_entry_frame0")[0]
    assert "fib__gtap_run(__frame, __tid, __ctx, __w0, __w1, true)" in out
    assert "__c->__dst = __gtap_dst(__tid, offsetof(__gtap_entry_frame0, __res));" in out
    assert "d_result = __f->__res;" in out


def test_parent_results_root_without_destination():
    out = lower_source(read("nq_pragma.cu"), results="parent")      # void tasks: no destination field
    frame = out[out.index("struct __gtap_frame_nq"):]
    assert "__dst" not in frame[:frame.index("};")]
    src = read("fib_pragma.cu").replace("    d_result = fib(n);", "    fib(n);")
    out = lower_source(src, results="parent")
    assert "__e->__dst = 0u;" in out                                # a root whose result goes nowhere


PARENT_BAD = {
    "block mode": ("tree_block_pragma.cu", None),
    "result into an array element": (None, """
#pragma gtap function
__device__ int f(int n, int* out) {
    if (n < 2) return n;
    #pragma gtap task
    out[0] = f(n - 1, out);
    #pragma gtap taskwait
    return out[0];
}
"""),
    "result of another type": (None, """
#pragma gtap function
__device__ int f(int n) {
    if (n < 2) return n;
    long long a;
    #pragma gtap task
    a = f(n - 1);
    #pragma gtap taskwait
    return (int)a;
}
"""),
    "two results into one local at one join": (None, """
#pragma gtap function
__device__ int f(int n) {
    if (n < 2) return n;
    int a;
    #pragma gtap task
    a = f(n - 1);
    #pragma gtap task
    a = f(n - 2);
    #pragma gtap taskwait
    return a;
}
"""),
    "return before the join": (None, """
#pragma gtap function
__device__ int f(int n) {
    if (n < 2) return n;
    int a;
    #pragma gtap task
    a = f(n - 1);
    if (n == 5) return 0;
    #pragma gtap taskwait
    return a;
}
"""),
}


@pytest.mark.parametrize("what", sorted(PARENT_BAD))
def test_parent_results_refusals(what):
    name, src = PARENT_BAD[what]
    with pytest.raises(LoweringError):
        lower_source(read(name) if name else src, results="parent")


@pytest.mark.skipif(shutil.which(NVCC) is None, reason="nvcc not available")
@pytest.mark.parametrize("src,defs", [
    ("fib_pragma.cu", "-DGTAP_MAX_CHILD_TASKS=2"),
    ("walk_pragma.cu", ""),
    ("fib_queues_pragma.cu", "-DGTAP_NUM_QUEUES=3"),
    ("cilksort_pragma.cu", ""),
    ("bary_tree_pragma.cu", "-DGTAP_MAX_CHILD_TASKS=8"),
])
def test_parent_results_programs_compile(tmp_path, src, defs):
    """Each compiles, and its kernel fits every worker on the GPU at once:
    888 blocks of 128 threads over 148 SMs is 6 blocks (768 threads) per SM,
    at most 65536 / 768 = 85 registers a thread; the bounds may spill a few
    registers."""
    low = tmp_path / ("parent_" + src)
    low.write_text(lower_source(read(src), results="parent"))
    cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-diag-suppress", "550",
           "-I", os.path.join(ROOT, "include"), "-DGTAP_GRID_SIZE=888", "-DGTAP_BLOCK_SIZE=128",
           "-Xptxas", "-v", "-c", str(low), "-o", str(tmp_path / "prog.o")] + defs.split()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = r.stderr.splitlines()
    k = next(i for i, ln in enumerate(lines) if "Function properties for _Z11exec_kernel" in ln)
    spilled = int(re.search(r"(\d+) bytes spill stores", lines[k + 1]).group(1))
    assert spilled <= 64, lines[k + 1]      # a few registers at most (three queues spill 20 bytes)
    regs = int(re.search(r"Used (\d+) registers", lines[k + 2]).group(1))
    assert regs <= 85, lines[k + 2]


@pytest.mark.skipif(shutil.which(NVCC) is None, reason="nvcc not available")
@pytest.mark.parametrize("src,defs", [
    ("fib_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2"),
    ("nq_pragma.cu", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("walk_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128"),
    ("fib_queues_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2 -DGTAP_NUM_QUEUES=3"),
    ("bary_tree_pragma.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=8"),
])
def test_default_lowering_keeps_every_worker_resident(tmp_path, src, defs):
    """The default (retained-result) lowering also bounds the entry kernel:
    GTAP_GRID_SIZE blocks over 148 SMs must all be resident, so the kernel
    may use at most 65536 / (threads per SM) registers a thread (1184 x 128
    threads: 64; 888 x 128: 85)."""
    out = lower_source(read(src))
    assert "__launch_bounds__(GTAP_BLOCK_SIZE" in out
    low = tmp_path / ("retain_" + src)
    low.write_text(out)
    cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-diag-suppress", "550",
           "-I", os.path.join(ROOT, "include"), "-Xptxas", "-v", "-c", str(low), "-o", str(tmp_path / "prog.o")]
    r = subprocess.run(cmd + defs.split(), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = r.stderr.splitlines()
    k = next(i for i, ln in enumerate(lines) if "Function properties for _Z11exec_kernel" in ln)
    regs = int(re.search(r"Used (\d+) registers", lines[k + 2]).group(1))
    grid = int(re.search(r"GTAP_GRID_SIZE=(\d+)", defs).group(1))
    threads_per_sm = -(-grid // 148) * 128
    assert regs * threads_per_sm <= 65536, (regs, threads_per_sm)
    spilled = int(re.search(r"(\d+) bytes spill stores", lines[k + 1]).group(1))
    assert spilled <= 64, lines[k + 1]
