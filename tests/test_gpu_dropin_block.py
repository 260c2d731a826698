"""Drop-in block-mode task ABI (include/gtap_block.cuh) on the GPU (B200 only).

Programs hand-lowered to the reference's block-mode task ABI
(tests/lowered/*_block_lowered.cu: the reference's block BFS, and a binary
tree in the shape of its block tree program with integer work) are compiled
against this repository's gtap_block.cuh and run as ordinary executables at
the reference's geometry (4000 blocks of 32 threads) and at a B200 geometry.
Their results must equal the oracle's / the closed form.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bins():
    from gtap_b200.build import build_lowered
    return {os.path.basename(p): p for p in build_lowered()}


def run(exe, *args, timeout=180):
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def tree_expect(height, work):
    nodes = np.arange(2 ** (height + 1) - 1, dtype=np.uint64)
    items = np.arange(work, dtype=np.uint64)
    v = ((nodes[:, None] * np.uint64(2654435761) + items[None, :] * np.uint64(40503)) % np.uint64(1 << 32)) >> np.uint64(22)
    return int(v.sum(dtype=np.uint64))


@pytest.mark.parametrize("name", ["tree_block_ref_geometry", "tree_block_b200"])
@pytest.mark.parametrize("height,work", [(0, 64), (1, 1), (6, 300), (12, 512)])
def test_tree_block_dropin(bins, name, height, work):
    r = run(bins[name], height, work, 3)
    assert r["error_code"] == 0
    assert r["result"] == tree_expect(height, work)


@pytest.mark.parametrize("name", ["bfs_block_ref_geometry", "bfs_block_b200"])
@pytest.mark.parametrize("scale", [8, 12, 15])
def test_bfs_block_dropin(bins, name, scale, tmp_path):
    out = tmp_path / "depth.bin"
    r = run(bins[name], scale, 42 + scale, 2, out)
    assert r["error_code"] == 0
    row, col = gt.gen_rmat(scale, 16, 42 + scale)
    src = gt.max_degree_vertex(row)
    assert r["source"] == src
    assert np.array_equal(np.fromfile(out, dtype=np.int32), orc.bfs(row, col, src))
