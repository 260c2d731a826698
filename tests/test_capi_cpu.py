"""C-ABI library checks that need no GPU: it loads, exports every entry point
include/gtap.h declares, and its host-side generators agree with the oracle."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import gtap_b200 as gt
from tests import oracle_lib as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    src = open(os.path.join(ROOT, "include", "gtap.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gtap_\w+)\s*\(", src)))


def test_library_builds_and_loads():
    L = gt.lib()
    assert gt.lib().gtap_version().decode().startswith("gtap_b200")


def test_exports_every_declared_symbol():
    names = declared_entry_points()
    assert len(names) >= 25
    L = ctypes.CDLL(gt.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert set(names) <= set(gt.EXPORTED)
    # dynamic symbol table really has them as global functions
    nm = subprocess.run(["nm", "-D", "--defined-only", gt.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT %s$" % n, nm, flags=re.M), n


def test_struct_layouts_match_header():
    # sizes the C side uses (checked through offsets of the last fields)
    assert ctypes.sizeof(gt.Root) == 56
    assert ctypes.sizeof(gt.RootResult) == 40
    assert gt.Config.total_ids.offset == 40
    assert gt.Config.admit_order.offset == 80 and gt.Config.leaf_batch.offset == 84
    assert gt.Config.join_walk.offset == 88 and gt.Config.sub_rounds.offset == 92
    assert ctypes.sizeof(gt.Config) == 96
    assert ctypes.sizeof(gt.RunStats) == 168
    assert gt.RunStats.light_kernel_ms.offset == 160


def test_default_config():
    c = gt.default_config()
    assert c.mode == gt.MODE_THREAD and c.block % 32 == 0
    assert c.num_queues == 1 and c.steal_batch == 32
    assert c.deque_capacity & (c.deque_capacity - 1) == 0
    assert c.join_walk == 0     # continuations resume as tasks unless a tuned configuration says otherwise
    assert c.sub_rounds == 0    # one pass of task bodies per round


def test_error_strings():
    assert gt.gtap_get_runtime_error_string(0) == "No error"
    assert gt.gtap_get_runtime_error_string(3) == "Queue overflow"
    assert gt.gtap_get_runtime_error_string(9) == "Timeout"


def test_calls_before_initialize_fail_cleanly():
    code = ctypes.c_int(0)
    assert gt.lib().gtap_get_runtime_error_code(ctypes.byref(code)) == gt.ERROR_NOT_INITIALIZED
    assert gt.lib().gtap_reset() == gt.ERROR_NOT_INITIALIZED
    r = (gt.Root * 1)(gt.fib_root(10))
    assert gt.lib().gtap_launch(r, 1, None, None, None) == gt.ERROR_NOT_INITIALIZED
    assert gt.lib().gtap_serve_poll(None, 0, None) == gt.ERROR_NOT_INITIALIZED


def test_invalid_config_rejected():
    c = gt.default_config(block=100)
    assert gt.lib().gtap_initialize(ctypes.byref(c)) == gt.ERROR_INVALID_ARGUMENT
    c = gt.default_config(deque_capacity=1000)
    assert gt.lib().gtap_initialize(ctypes.byref(c)) == gt.ERROR_INVALID_ARGUMENT
    c = gt.default_config(num_queues=5)
    assert gt.lib().gtap_initialize(ctypes.byref(c)) == gt.ERROR_INVALID_ARGUMENT
    # rounds that walk fib's sums at their joins: 0..32 tasks; extra passes on idle lanes: 0..8
    for field, bad in (("join_walk", -1), ("join_walk", 33), ("sub_rounds", -1), ("sub_rounds", 9)):
        c = gt.default_config(**{field: bad})
        assert gt.lib().gtap_initialize(ctypes.byref(c)) == gt.ERROR_INVALID_ARGUMENT, (field, bad)


def test_gen_keys_matches_oracle_and_std():
    for seed, n in [(42, 1000), (1, 1 << 16), (5489, 10000)]:
        assert np.array_equal(gt.gen_keys(seed, n), orc.keys(seed, n))


def test_gen_mix_matches_oracle():
    a = gt.gen_mix(42, 4096)
    b = orc.root_mix(42, 4096)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_gen_rmat_matches_oracle():
    r1, c1 = gt.gen_rmat(11, 16, 42)
    r2, c2 = orc.rmat(11, 16, 42)
    assert np.array_equal(r1, r2) and np.array_equal(c1, c2)
    assert r1[-1] == 16 << 11
    assert gt.max_degree_vertex(r1) == orc.max_degree_vertex(r2)


def test_gen_tree_matches_oracle():
    a = gt.gen_tree(20000, 9)
    b = orc.tree(20000, 9)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_generator_argument_checks():
    assert gt.lib().gtap_gen_keys(1, None, 10) == gt.ERROR_INVALID_ARGUMENT
    assert gt.lib().gtap_gen_rmat(0, 16, 1, None, None) == gt.ERROR_INVALID_ARGUMENT
