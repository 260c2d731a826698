"""Programs written with the gtap pragmas (tests/pragma), lowered by
gtap_b200.lower and run on the B200 (B200 only): results must equal the
oracle's (fib, n-queens), the sort must be ascending and a permutation of its
input, and the block-mode tree sum must equal its closed form."""
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


@pytest.mark.parametrize("n,cutoff", [(0, 0), (1, 0), (2, 0), (20, 0), (27, 0), (30, 12)])
def test_fib_pragma(bins, n, cutoff):
    r = run(bins["fib_pragma"], n, cutoff, 2)
    assert r["error_code"] == 0
    assert r["results"] == [orc.fib(n)] * 2


@pytest.mark.parametrize("n,cutoff", [(4, 3), (8, 7), (10, 4), (12, 6)])
def test_nq_pragma(bins, n, cutoff):
    r = run(bins["nq_pragma"], n, cutoff)
    assert r["error_code"] == 0
    assert r["result"] == orc.nq(n)


@pytest.mark.parametrize("n", [1, 63, 1000, 100003, 1 << 20])
def test_cilksort_pragma(bins, n):
    r = run(bins["cilksort_pragma"], n, 7)
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
