"""Programs written with the gtap pragmas (tests/pragma), lowered by
gtap_b200.lower and run on the B200 (B200 only): results must equal the
oracle's (fib, n-queens), the sort must be ascending and a permutation of its
input (thread-mode programs also in the --results parent lowering), the block-mode tree sum must equal its closed form, and the ternary
walk (taskwaits inside if/else branches) must equal its recursion in Python;
the probabilistic B-ary tree's mix sum and node count must equal the oracle's,
in thread mode and in block mode."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests import oracle_lib as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bins():
    from gtap_b200.build import build_pragma
    return {os.path.basename(p): p for p in build_pragma()}


def run(exe, *args, timeout=180):
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


# "_parent": the same program lowered with --results parent (children write
# their results into the parent's frame)
VARIANTS = ["", "_parent"]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("n,cutoff", [(0, 0), (1, 0), (2, 0), (20, 0), (27, 0), (30, 0), (30, 12)])
def test_fib_pragma(bins, n, cutoff, variant):
    r = run(bins["fib_pragma" + variant], n, cutoff, 2)
    assert r["error_code"] == 0
    assert r["results"] == [orc.fib(n)] * 2


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("n,cutoff", [(0, 0), (2, 0), (22, 0), (29, 0), (32, 14)])
def test_fib_queues_pragma(bins, n, cutoff, variant):
    r = run(bins["fib_queues_pragma" + variant], n, cutoff, 2)
    assert r["error_code"] == 0 and r["queues"] == 3
    assert r["results"] == [orc.fib(n)] * 2


@pytest.mark.parametrize("n,cutoff", [(4, 3), (8, 7), (10, 4), (12, 6)])
def test_nq_pragma(bins, n, cutoff):
    r = run(bins["nq_pragma"], n, cutoff)
    assert r["error_code"] == 0
    assert r["result"] == orc.nq(n)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("n", [1, 63, 1000, 100003, 1 << 20])
def test_cilksort_pragma(bins, n, variant):
    r = run(bins["cilksort_pragma" + variant], n, 7)
    assert r["error_code"] == 0
    assert r["sorted"] is True


def tree_expect(height, work):
    nodes = np.arange(2 ** (height + 1) - 1, dtype=np.uint64)
    items = np.arange(work, dtype=np.uint64)
    v = ((nodes[:, None] * np.uint64(2654435761) + items[None, :] * np.uint64(40503)) % np.uint64(1 << 32)) >> np.uint64(22)
    return int(v.sum(dtype=np.uint64))


@pytest.mark.parametrize("height,work", [(0, 10), (3, 100), (10, 300)])
def test_tree_block_pragma(bins, height, work):
    r = run(bins["tree_block_pragma"], height, work)
    assert r["error_code"] == 0
    assert r["result"] == tree_expect(height, work)


M64 = (1 << 64) - 1


def walk_expect(depth, ident):
    """walk_pragma.cu's walk() evaluated on the CPU, modulo 2^64."""
    k = ident % 3
    a = b = 0
    own = ident
    scale = depth * 7 + 1
    if depth == 0:
        return own * scale & M64
    if k == 0:
        a = walk_expect(depth - 1, 3 * ident + 1)
        b = walk_expect(depth - 1, 3 * ident + 2)
        own = (own + a - b) & M64
    else:
        own += ident & 7
        if k == 1:
            a = walk_expect(depth - 1, 3 * ident + 1)
        walk_expect(depth - 1, 3 * ident + 2)
        own = (own + 2 * a + k) & M64
    b = walk_expect(depth // 2, ident + 1)
    return (own * scale + b) & M64


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("depth,ident", [(0, 5), (1, 0), (1, 1), (1, 2), (6, 0), (9, 1), (11, 2), (16, 0), (16, 4)])
def test_walk_pragma(bins, depth, ident, variant):
    r = run(bins["walk_pragma" + variant], depth, ident)
    assert r["error_code"] == 0
    assert r["result"] == walk_expect(depth, ident)


@pytest.mark.parametrize("D,B,mem_ops,iters,log2n", [
    (0, 3, 4, 4, 10), (1, 3, 4, 4, 10), (6, 3, 8, 16, 12), (9, 4, 16, 32, 16), (15, 4, 8, 8, 16),
    (18, 4, 16, 64, 22),
])
@pytest.mark.parametrize("variant", VARIANTS)
def test_bary_tree_pragma(bins, D, B, mem_ops, iters, log2n, variant):
    seed = 7 + D
    r = run(bins["bary_tree_pragma" + variant], D, B, mem_ops, iters, log2n, seed, 2)
    assert r["error_code"] == 0
    total, nodes = orc.bary_tree(D, B, mem_ops, iters, orc.bary_input(seed, 1 << log2n))
    assert r["nodes"] == nodes
    assert r["sum"] == total


@pytest.mark.parametrize("D,B,mem_ops,iters,log2n", [
    (0, 3, 4, 4, 10), (1, 3, 300, 200, 10), (6, 3, 64, 256, 12), (9, 4, 300, 200, 16), (13, 4, 128, 512, 20),
])
def test_bary_block_pragma(bins, D, B, mem_ops, iters, log2n):
    seed = 11 + D
    r = run(bins["bary_block_pragma"], D, B, mem_ops, iters, log2n, seed, 2)
    assert r["error_code"] == 0
    total, nodes = orc.bary_tree_block(D, B, mem_ops, iters, r["threads"], orc.bary_input(seed, 1 << log2n))
    assert r["nodes"] == nodes
    assert r["sum"] == total
