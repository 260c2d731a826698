"""Seeded workloads used by the benchmark and the autotuner.

The batched mix: `gtap_gen_mix(seed, n)` draws n roots, kind uniform over
{fib, n-queens, cilksort}; fib n in [18, 28] without cutoff, n-queens n in
[8, 11] with one task per row, cilksort of m * 2^e int32 keys with m uniform
in [1024, 2048) and e uniform in [0, 9] (so sizes span 2^10 .. 2^20, log-
uniform by octave), keys = std::mt19937(per-root seed).  All cilksort roots share three
device slabs (source, sorted output, scratch); the leaves read the source, so
a repeated launch needs no restore.
"""
import numpy as np

MIX_SEED = 42
N_ROOTS = 4096
SORT_CUTOFF, MERGE_CUTOFF = 64, 256   # examples/cilksort/cilksort.cu:10-11


class Mix:
    """The seeded root mix.  `gen` supplies gen_mix(seed, n) and
    gen_keys(seed, n): the library module (gtap_b200) or any object with the
    same two generators."""

    def __init__(self, gen, n_roots=N_ROOTS, seed=MIX_SEED):
        gt = gen
        self.kind, self.param, self.seed = gt.gen_mix(seed, n_roots)
        sizes = np.where(self.kind == 2, self.param, 0).astype(np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(sizes)])
        self.total_keys = int(self.offsets[-1])
        keys = np.empty(max(self.total_keys, 1), np.int32)
        for i in np.nonzero(self.kind == 2)[0]:
            o, n = int(self.offsets[i]), int(self.param[i])
            keys[o:o + n] = gt.gen_keys(int(self.seed[i]) & 0xFFFFFFFF, n)
        self.keys = keys
        self.n = n_roots

    def roots(self, gt, src, arr, tmp, elem=4):
        """Root descriptors over slabs at addresses src / arr / tmp."""
        rs = []
        for i in range(self.n):
            k, p = int(self.kind[i]), int(self.param[i])
            if k == 0:
                rs.append(gt.fib_root(p, 0))
            elif k == 1:
                rs.append(gt.nq_root(p))
            else:
                o = int(self.offsets[i]) * elem
                rs.append(gt.cilksort_root(src + o, arr + o, tmp + o, p, SORT_CUTOFF, MERGE_CUTOFF))
        return rs

    def device_slabs(self):
        """(src, arr, tmp) torch tensors on the current device."""
        import torch
        src = torch.from_numpy(self.keys).cuda()
        return src, torch.empty_like(src), torch.empty_like(src)


def single_root_workload(gt, name):
    """fib30 / nq13 / fib34c12: the single-root configurations, as root lists."""
    table = {
        "fib30": [gt.fib_root(30, 0)],
        "fib34c12": [gt.fib_root(34, 12)],
        "nq13": [gt.nq_root(13)],
        "nq13c7": [gt.nq_root(13, 7)],
    }
    return table[name]
