"""The drop-in task-ABI headers (include/gtap_thread.cuh, include/gtap_block.cuh)
compile for sm_100a with lowered reference programs, without a GPU: nvcc
builds the objects only (the GPU tests link and run them)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "nvcc")


@pytest.mark.skipif(shutil.which(NVCC) is None, reason="nvcc not available")
@pytest.mark.parametrize("src,defs", [
    ("fib_lowered.cu", "-DGTAP_GRID_SIZE=888 -DGTAP_BLOCK_SIZE=128 -DGTAP_MAX_CHILD_TASKS=2"),
    ("nq_lowered.cu", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128 -DGTAP_ASSUME_NO_TASKWAIT"),
    ("tree_block_lowered.cu", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=128"),
    ("bfs_block_lowered.cu", "-DGTAP_GRID_SIZE=1184 -DGTAP_BLOCK_SIZE=256 -DGTAP_ASSUME_NO_TASKWAIT"),
])
def test_lowered_program_compiles(tmp_path, src, defs):
    cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-diag-suppress", "550",
           "-I", os.path.join(ROOT, "include"), "-c", os.path.join(ROOT, "tests", "lowered", src),
           "-o", str(tmp_path / "prog.o")] + defs.split()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    assert (tmp_path / "prog.o").stat().st_size > 0
