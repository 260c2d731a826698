"""Admission order of a batch launch (host side, no device call): the stable
grouping by kind that GTAP_ADMIT_BY_KIND and GTAP_ADMIT_SPLIT admit roots in,
and the split point of a split batch.  The device side (results returned in the
caller's order, the same values and task counts under every admission order)
is covered by tests/test_gpu_admission.py."""
import numpy as np
import pytest

import gtap_b200 as gt

FIB, NQ, CILKSORT, MERGESORT, BFS, TREESUM = 1, 2, 3, 4, 5, 6
# group rank: invalid kinds, then the kinds without sort leaves in kind order, then the sorts
RANK = {FIB: 1, NQ: 2, BFS: 5, TREESUM: 6, CILKSORT: 10, MERGESORT: 11}


def _roots(kinds):
    out = []
    for i, k in enumerate(kinds):
        r = gt.Root()
        r.kind, r.i0 = int(k), i
        out.append(r)
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_grouping_is_stable_and_puts_sorts_last(seed):
    rng = np.random.default_rng(seed)
    kinds = rng.choice([FIB, NQ, CILKSORT, MERGESORT, BFS, TREESUM], size=777)
    order, n_light = gt.admission_order(_roots(kinds))
    assert sorted(order) == list(range(len(kinds)))
    ranks = [RANK[int(kinds[i])] for i in order]
    assert ranks == sorted(ranks)
    # stable: within a kind, the caller's order
    for k in RANK:
        idx = [i for i in order if kinds[i] == k]
        assert idx == sorted(idx)
    assert n_light == int(np.sum((kinds != CILKSORT) & (kinds != MERGESORT)))
    assert all(kinds[i] in (CILKSORT, MERGESORT) for i in order[n_light:])


def test_invalid_kinds_lead():
    kinds = [CILKSORT, 0, FIB, 99, NQ, -3]
    order, n_light = gt.admission_order(_roots(kinds))
    assert order == [1, 3, 5, 2, 4, 0]
    assert n_light == 5


def test_grouped_batch_keeps_its_order():
    kinds = [FIB] * 5 + [NQ] * 3 + [BFS] + [CILKSORT] * 4 + [MERGESORT]
    order, n_light = gt.admission_order(_roots(kinds))
    assert order == list(range(len(kinds)))
    assert n_light == 9


def test_single_kind_batches():
    for k in (FIB, CILKSORT):
        order, n_light = gt.admission_order(_roots([k] * 10))
        assert order == list(range(10))
        assert n_light == (10 if k == FIB else 0)
    assert gt.admission_order([]) == ([], 0)


def test_admit_order_is_validated():
    c = gt.default_config()
    assert c.admit_order == gt.ADMIT_SPLIT
    # rejected before any device work
    for bad in (-1, 3):
        c.admit_order = bad
        with pytest.raises(gt.GtapError):
            gt.gtap_initialize(c)
