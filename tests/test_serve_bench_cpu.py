"""The serve benchmark's BFS validation on the CPU: it accepts the oracle's
distance labelling and rejects labellings with one level wrong or one vertex
dropped."""
import numpy as np
import pytest

import gtap_b200 as gt
from gtap_b200.serve_bench import INF, bfs_depths_valid
from tests import oracle_lib as orc


@pytest.mark.parametrize("scale", [6, 10, 12])
def test_bfs_validation(scale):
    row, col = gt.gen_rmat(scale, 16, 5 + scale)
    src = gt.max_degree_vertex(row)
    d = orc.bfs(row, col, src)
    assert bfs_depths_valid(row, col, src, d)
    reached = np.nonzero((d < INF) & (np.arange(len(d)) != src))[0]
    off = d.copy()
    off[reached[len(reached) // 2]] += 1
    assert not bfs_depths_valid(row, col, src, off)
    dropped = d.copy()
    dropped[reached[-1]] = INF
    assert not bfs_depths_valid(row, col, src, dropped)
    moved = d.copy()
    moved[src] = 1
    assert not bfs_depths_valid(row, col, src, moved)
