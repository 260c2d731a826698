"""The oracle's probabilistic B-ary tree (oracle/oracle.c, orc_bary_*) pinned
on the CPU: its hash and input generator against their published test
vectors, and the node work and tree against an independent restatement in
Python whose fused multiply-add is exact rational arithmetic rounded once."""
from fractions import Fraction
import struct

import numpy as np

from tests import oracle_lib as orc

M32 = 0xFFFFFFFF
M64 = (1 << 64) - 1


def fmix32(h):
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & M32
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & M32
    return h ^ (h >> 16)


def fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))   # one rounding: int / int is correctly rounded


def node_work(node, inp, mem_ops, iters):
    seed = fmix32(node ^ 0x2545F491)
    acc = 0.0
    for m in range(mem_ops):
        acc += float(inp[fmix32((seed + m) & M32) & (len(inp) - 1)])
    mix = ((seed ^ 0x9E3779B9) + (int(acc) & M32)) & M32      # int() truncates toward zero, as C does
    y = 0.0
    for it in range(iters):
        x = float(fmix32((seed + it * 0x632BE5AB) & M32))
        y = fma(x, 1.0000001192092896, y)
        bits = struct.unpack("<Q", struct.pack("<d", y))[0]
        mix ^= (bits & M32) ^ (bits >> 32)
    return mix


def tree(D, B, mem_ops, iters, inp):
    total, count, stack = 0, 0, [(0, 0)]
    while stack:
        node, d = stack.pop()
        if d < D:
            s = fmix32(node ^ ((d * 0x9E3779B9) & M32))
            for k in range(B):
                s = fmix32((s + k) & M32)
                if s % D < D - d:
                    stack.append(((node * B + k + 1) & M32, d + 1))
        total = (total + node_work(node, inp, mem_ops, iters)) & M64
        count += 1
    return total, count


def test_published_vectors():
    L = orc.load()
    assert L.orc_fmix32(0) == 0 and L.orc_fmix32(1) == 0x514E28B7    # MurmurHash3 fmix32
    first = orc.bary_input(0, 1)[0]                                   # splitmix64(0) = 0xe220a8397b1dcdaf
    assert first == (0xE220A8397B1DCDAF >> 11) * 2.0 ** -53 * 2.0 - 1.0


def test_input_range():
    inp = orc.bary_input(7, 1 << 14)
    assert inp.min() >= -1.0 and inp.max() < 1.0 and abs(inp.mean()) < 0.05


def test_node_work_matches_exact_restatement():
    inp = orc.bary_input(11, 1 << 12)
    L = orc.load()
    for node in [0, 1, 2, 3, 17, 1000, 123456789, M32]:
        for mem_ops, iters in [(0, 0), (4, 4), (16, 40)]:
            assert L.orc_bary_node_work(node, orc.p(inp), len(inp), mem_ops, iters) == node_work(node, inp, mem_ops, iters)


def test_tree_matches_exact_restatement():
    inp = orc.bary_input(3, 1 << 10)
    for D, B, mem_ops, iters in [(0, 3, 2, 2), (1, 3, 4, 4), (4, 3, 8, 8), (6, 2, 3, 5)]:
        assert orc.bary_tree(D, B, mem_ops, iters, inp) == tree(D, B, mem_ops, iters, inp)


def test_spawn_probability_follows_depth():
    # root: all B children; the last level keeps about 1/D of its candidates
    D, B = 8, 4
    assert orc.bary_tree(1, B, 0, 0, orc.bary_input(1, 16))[1] == 1 + B
    kept = [0] * D
    tried = [0] * D
    stack = [(0, 0)]
    while stack:
        node, d = stack.pop()
        if d < D:
            s = fmix32(node ^ ((d * 0x9E3779B9) & M32))
            for k in range(B):
                s = fmix32((s + k) & M32)
                tried[d] += 1
                if s % D < D - d:
                    kept[d] += 1
                    stack.append(((node * B + k + 1) & M32, d + 1))
    for d in range(D):
        if tried[d] >= 200:
            assert abs(kept[d] / tried[d] - (D - d) / D) < 0.08


def node_work_block(node, inp, mem_ops, iters, threads):
    seed = fmix32(node ^ 0x2545F491)
    acc, xr = 0.0, 0
    for t in range(threads):
        part = 0.0
        for m in range(t, mem_ops, threads):
            part += float(inp[fmix32((seed + m) & M32) & (len(inp) - 1)])
        acc += part
        y = 0.0
        for it in range(t, iters, threads):
            y = fma(float(fmix32((seed + it * 0x632BE5AB) & M32)), 1.0000001192092896, y)
            bits = struct.unpack("<Q", struct.pack("<d", y))[0]
            xr ^= (bits & M32) ^ (bits >> 32)
    return (((seed ^ 0x9E3779B9) + (int(acc) & M32)) & M32) ^ xr


def test_block_node_work_matches_exact_restatement():
    inp = orc.bary_input(5, 1 << 12)
    L = orc.load()
    for node in [0, 9, 77777, M32]:
        for mem_ops, iters, threads in [(0, 0, 32), (5, 3, 4), (300, 200, 128), (64, 512, 128)]:
            assert (L.orc_bary_node_work_block(node, orc.p(inp), len(inp), mem_ops, iters, threads)
                    == node_work_block(node, inp, mem_ops, iters, threads))


def test_block_tree_has_the_thread_tree_shape():
    inp = orc.bary_input(9, 1 << 10)
    for D, B in [(0, 2), (5, 3), (8, 4)]:
        assert orc.bary_tree_block(D, B, 4, 4, 32, inp)[1] == orc.bary_tree(D, B, 4, 4, inp)[1]
