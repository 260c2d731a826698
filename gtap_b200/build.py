"""Build libgtap_b200.so in-tree with nvcc for sm_100a.

Usage: python -m gtap_b200.build  (or gtap_b200.build.build())
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgtap_b200.so")
LIB_DEBUG = os.path.join(HERE, "libgtap_b200_debug.so")

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared",
    "-diag-suppress", "550",
]


def sources():
    return [os.path.join(CSRC, "gtap_capi.cu"), os.path.join(CSRC, "gtap_noalloc.cu"),
            os.path.join(CSRC, "gtap_microbench.cu")]


LOWERED = os.path.join(ROOT, "tests", "lowered")
LOWERED_BIN = os.path.join(LOWERED, "bin")

# Programs lowered to the reference's task ABI, built against the drop-in
# headers include/gtap_thread.cuh and (block mode) include/gtap_block.cuh:
# (source, binary, -D settings).  "ref" builds use the reference's own
# evaluation settings, "b200" builds a geometry for 148 SMs.
LOWERED_BUILDS = [
    ("fib_lowered.cu", "fib_ref_geometry",
     "-DGTAP_GRID_SIZE=4000 -DGTAP_BLOCK_SIZE=32 -DGTAP_MAX_CHILD_TASKS=2"),
    ("fib_lowered.cu", "fib_b200",
     "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2"),
    ("nq_lowered.cu", "nq_ref_geometry",
     "-DGTAP_GRID_SIZE=2000 -DGTAP_BLOCK_SIZE=32 -DGTAP_MAX_CHILD_TASKS=32 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("nq_lowered.cu", "nq_b200",
     "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=32 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("cilksort_lowered.cu", "cilksort_ref_geometry",
     "-DGTAP_GRID_SIZE=2000 -DGTAP_BLOCK_SIZE=32 -DGTAP_MAX_CHILD_TASKS=7"),
    ("cilksort_lowered.cu", "cilksort_b200",
     "-DGTAP_GRID_SIZE=592 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=7"),
    ("bfs_block_lowered.cu", "bfs_block_ref_geometry",
     "-DGTAP_GRID_SIZE=4000 -DGTAP_BLOCK_SIZE=32 -DGTAP_MAX_TASKS_PER_BLOCK=150000 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("bfs_block_lowered.cu", "bfs_block_b200",
     "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=256 -DGTAP_MAX_TASKS_PER_BLOCK=20000 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("tree_block_lowered.cu", "tree_block_ref_geometry", "-DGTAP_GRID_SIZE=4000 -DGTAP_BLOCK_SIZE=32"),
    ("tree_block_lowered.cu", "tree_block_b200", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128"),
]


PRAGMA_DIR = os.path.join(ROOT, "tests", "pragma")
PRAGMA_BIN = os.path.join(PRAGMA_DIR, "bin")

# Programs written with the gtap pragmas, lowered by gtap_b200.lower and then
# compiled like the hand-lowered ones: (source, binary, -D settings).
PRAGMA_BUILDS = [
    ("fib_pragma.cu", "fib_pragma", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2"),
    ("nq_pragma.cu", "nq_pragma", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("cilksort_pragma.cu", "cilksort_pragma", "-DGTAP_GRID_SIZE=592 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=4"),
    ("tree_block_pragma.cu", "tree_block_pragma", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128"),
    ("walk_pragma.cu", "walk_pragma", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128"),
    ("bary_tree_pragma.cu", "bary_tree_pragma",
     "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=8"),
    ("bary_block_pragma.cu", "bary_block_pragma", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128"),
    ("fib_queues_pragma.cu", "fib_queues_pragma",
     "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2 -DGTAP_NUM_QUEUES=3"),
    # the same thread-mode programs lowered with results delivered into the
    # parent's frame (lower.py --results parent)
    ("fib_pragma.cu", "fib_pragma_parent", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2",
     "parent"),
    ("walk_pragma.cu", "walk_pragma_parent", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128", "parent"),
    ("fib_queues_pragma.cu", "fib_queues_pragma_parent",
     "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2 -DGTAP_NUM_QUEUES=3", "parent"),
    ("cilksort_pragma.cu", "cilksort_pragma_parent",
     "-DGTAP_GRID_SIZE=592 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=4", "parent"),
    ("bary_tree_pragma.cu", "bary_tree_pragma_parent",
     "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=8", "parent"),
]


def build_pragma(force=False):
    """Lower and compile the pragma programs (tests/pragma/*.cu) against the
    drop-in headers, linking libgtap_b200.so.  Returns the binaries' paths."""
    from gtap_b200.lower import lower_source
    build()
    os.makedirs(PRAGMA_BIN, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    header_deps = deps() + [os.path.join(HERE, "lower.py")]
    outs = []
    for entry in PRAGMA_BUILDS:
        src, name, defs = entry[:3]
        results = entry[3] if len(entry) > 3 else "retain"
        s = os.path.join(PRAGMA_DIR, src)
        out = os.path.join(PRAGMA_BIN, name)
        outs.append(out)
        if (not force and os.path.exists(out)
                and all(os.path.getmtime(p) <= os.path.getmtime(out) for p in header_deps + [s, LIB])):
            continue
        low = os.path.join(PRAGMA_BIN, name + "_lowered.cu")
        with open(s) as f:
            text = lower_source(f.read(), results=results)
        with open(low, "w") as f:
            f.write(text)
        cmd = ([nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
                "-diag-suppress", "550", "-I", os.path.join(ROOT, "include")] + defs.split()
               + ["-o", out, low, "-L", HERE, "-lgtap_b200", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../../gtap_b200"])
        r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed building %s" % name)
    return outs


def deps():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                out.append(os.path.join(d, f))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force=False, verbose=False, debug=False):
    """Compile the library; debug=True builds libgtap_b200_debug.so with
    per-task-id live checks (every violation is reported as a runtime error)."""
    out = LIB_DEBUG if debug else LIB
    if not force and not debug and up_to_date():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = ([nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + (["-DGTAP_DEBUG_IDS"] if debug else [])
           + ["-o", out] + sources())
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libgtap_b200.so")
    if verbose:
        sys.stderr.write(r.stderr)
    return out


def build_lowered(force=False, verbose=False):
    """Compile the lowered programs against include/gtap_thread.cuh, linking
    libgtap_b200.so (built first).  Returns the binaries' paths."""
    build(verbose=verbose)
    os.makedirs(LOWERED_BIN, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    header_deps = deps()
    outs = []
    for src, name, defs in LOWERED_BUILDS:
        s = os.path.join(LOWERED, src)
        out = os.path.join(LOWERED_BIN, name)
        outs.append(out)
        if (not force and os.path.exists(out)
                and all(os.path.getmtime(p) <= os.path.getmtime(out) for p in header_deps + [s, LIB])):
            continue
        cmd = ([nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
                "-diag-suppress", "550", "-I", os.path.join(ROOT, "include")] + defs.split()
               + ["-o", out, s, "-L", HERE, "-lgtap_b200", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../../gtap_b200"])
        r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed building %s" % name)
    return outs


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, debug="--debug" in sys.argv))
    if "--lowered" in sys.argv:
        print("\n".join(build_lowered(force="--force" in sys.argv)))
