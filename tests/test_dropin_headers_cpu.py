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


HELPERS = r'''
#include <stdint.h>
#include "%s"

__device__ int g_i[64];
__device__ unsigned g_u[64];
__device__ uint16_t g_h[64];
__device__ int* g_p[4];
__device__ unsigned long long g_out[8];

__device__ void helper_task(void* frame, int tid, TaskContext* ctx) {
    (void)frame;
    int a = load_L2(&g_i[1]) + load_L2_acquire(&g_i[2]);
    unsigned b = load_L2(&g_u[3]) + load_L2_u16t(&g_h[4]);
    int* p = load_L2_ptr(&g_p[0]);
    void* q = load_L2_ptr(reinterpret_cast<void**>(&g_p[1]));
    store_L2(&g_i[5], a);
    store_L2(&g_u[6], b);
    store_L2_u16t(&g_h[7], (uint16_t)b);
    store_L2_release(&g_i[8], a);
    store_L2_ptr(&g_p[2], p);
    store_L2_ptr(reinterpret_cast<void**>(&g_p[3]), q);
    int old = atomicCAS_acquire(&g_i[9], 0, 1);
    g_out[0] = get_lane_id() + get_warp_id_in_block() + get_warp_id_global() + (unsigned)old;
    g_out[1] = get_global_time();
    __gtap_finish_task(tid, ctx);
}

const size_t __gtap_auto_task_data_size = 16;

__global__ void exec_kernel() {
    if (blockIdx.x == 0 && threadIdx.x == 0) __gtap_push_initial_task(helper_task, 0);
    __gtap_execute_task_loop_device();
}
'''


@pytest.mark.skipif(shutil.which(NVCC) is None, reason="nvcc not available")
@pytest.mark.parametrize("header", ["gtap_thread.cuh", "gtap_block.cuh"])
def test_device_helpers_compile_in_task_code(tmp_path, header):
    """Every helper of include/gtap_device_util.cuh (the reference's load_L2 /
    store_L2 family, lane and warp ids, the global timer) used from a task."""
    src = tmp_path / "helpers.cu"
    src.write_text(HELPERS % header)
    cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-diag-suppress", "550",
           "-I", os.path.join(ROOT, "include"), "-DGTAP_GRID_SIZE=148", "-DGTAP_BLOCK_SIZE=128",
           "-c", str(src), "-o", str(tmp_path / "helpers.o")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
