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
    return [os.path.join(CSRC, "gtap_capi.cu"), os.path.join(CSRC, "gtap_noalloc.cu")]


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


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, debug="--debug" in sys.argv))
