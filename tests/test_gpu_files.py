"""The reference's on-disk inputs on the GPU path (B200 only).

The reference's programs read their inputs from files: cilksort and mergesort
an int32 array in gen_vector's format (size_t n, then n int32;
evaluation/util/gen_vector.c:21-36), asynchronous BFS a CSR binary (int N,
int M, row[N+1], col[M]; examples/asynchronous_bfs/asynchronous_bfs_thread.cu:
69-84).  Here such files are written with the library's writers, read back
with its loaders, and the arrays they yield are sorted or searched on the
device; every output must equal the oracle's on the same data, and the files'
bytes must be exactly the format above.
"""
import struct

import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu

INF = 0x3f3f3f3f


@pytest.mark.parametrize("mode,n,cut", [(gt.MODE_THREAD, 100_003, (64, 256)), (gt.MODE_THREAD, 1 << 20, (64, 256)),
                                         (gt.MODE_BLOCK, 3_000_017, (2048, 2048))])
def test_sort_a_gen_vector_file(tmp_path, mode, n, cut):
    import torch
    keys = orc.keys(1234 + n, n)
    path = tmp_path / "vec.bin"
    gt.write_array(path, keys)
    raw = path.read_bytes()
    assert struct.unpack("<Q", raw[:8])[0] == n and len(raw) == 8 + 4 * n   # size_t n, then n int32
    loaded = gt.read_array(path)
    assert np.array_equal(loaded, keys)
    src = torch.from_numpy(loaded).cuda()
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    gt.gtap_initialize(gt.default_config(mode=mode))
    try:
        res, st = gt.launch([gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, *cut)])
    finally:
        gt.gtap_finalize()
    assert res[0].status == gt.ROOT_DONE and st.status == 0
    want, s_tasks, m_tasks = orc.cilksort(keys, *cut)
    assert np.array_equal(arr.cpu().numpy(), want)
    assert res[0].tasks == s_tasks + m_tasks


def test_mergesort_a_gen_vector_file_through_host_buffers(tmp_path):
    """The host-buffer entry point on a loaded file: keys copied in, sorted
    keys copied back into the caller's buffer."""
    n = 500_000
    keys = orc.keys(99, n)
    path = tmp_path / "vec.bin"
    gt.write_array(path, keys)
    host_in = gt.read_array(path)
    host_out = np.empty_like(host_in)
    gt.gtap_initialize(gt.default_config())
    try:
        res, st, h2d, d2h = gt.run_host([gt.mergesort_root(host_in.ctypes.data, host_out.ctypes.data, 0, n, 128)])
    finally:
        gt.gtap_finalize()
    assert res[0].status == gt.ROOT_DONE
    assert np.array_equal(host_out, orc.sort(keys))
    assert h2d >= 4 * n and d2h >= 4 * n


@pytest.mark.parametrize("mode,scale", [(gt.MODE_THREAD, 14), (gt.MODE_THREAD, 17), (gt.MODE_BLOCK, 16)])
def test_bfs_on_a_csr_file(tmp_path, mode, scale):
    import torch
    row, col = orc.rmat(scale, 16, 500 + scale)
    path = tmp_path / "graph.csr"
    gt.write_csr(path, row, col)
    raw = path.read_bytes()
    nv, ne = struct.unpack("<ii", raw[:8])
    assert (nv, ne) == (len(row) - 1, len(col)) and len(raw) == 8 + 4 * (nv + 1) + 4 * ne
    r2, c2 = gt.read_csr(path)
    assert np.array_equal(r2, row) and np.array_equal(c2, col)
    src = orc.max_degree_vertex(r2)
    drow, dcol = torch.from_numpy(r2).cuda(), torch.from_numpy(c2).cuda()
    depth = torch.full((nv,), INF, dtype=torch.int32, device="cuda")
    gt.gtap_initialize(gt.default_config(mode=mode))
    try:
        res, st = gt.launch([gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), depth.data_ptr(), nv, src, 32)])
    finally:
        gt.gtap_finalize()
    assert res[0].status == gt.ROOT_DONE and st.status == 0
    assert np.array_equal(depth.cpu().numpy(), orc.bfs(row, col, src))
