"""One root launched a few times, for profiler captures of a single worker
kernel on a small case.

    python -m gtap_b200.profile_case mergesort   # thread mode, 2^24 keys, cutoffs 128 / 256
    python -m gtap_b200.profile_case cilksort_block   # block mode, 2^25 keys, cutoffs 2048 / 2048
    python -m gtap_b200.profile_case fib30       # thread mode, fib(30) without cutoff

Keys are std::mt19937(42) draws (gtap_gen_keys), the arena holds 2^22 task
records (enough for these trees, and a few hundred MB for a profiler to save
and restore between passes), and every launch's output must equal a device
sort of the keys (fib: the value and task count of the recursion).  The configuration is the tuner's file for the workload when
it exists (the library defaults otherwise).  Each launch prints its CUDA-event
time: under a profiler those are not measurements.
"""
import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = {
    # name: (keys, mode, tuned file)
    "mergesort": (1 << 24, "thread", "b200_mergesort24.json"),
    "cilksort_block": (1 << 25, "block", "b200_cilksort26_block.json"),
    "fib30": (30, "thread", "b200_fib30.json"),
}


def fib_value_and_tasks(n):
    """fib(n) and the tasks of its call tree without cutoff (2 fib(n+1) - 1)."""
    a, b = 0, 1
    for _ in range(n):
        a, b = b, a + b
    return a, 2 * b - 1


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--launches", type=int, default=3)
    a = ap.parse_args(argv)
    import torch
    import gtap_b200 as gt
    from gtap_b200.autotune import load_tuned
    n, mode, tuned = CASES[a.case]
    over = load_tuned(os.path.join(ROOT, "gtap_b200", "tuned", tuned))
    over["total_ids"] = 1 << 22
    over["mode"] = gt.MODE_BLOCK if mode == "block" else gt.MODE_THREAD
    gt.gtap_initialize(gt.default_config(**over))
    try:
        if a.case == "fib30":
            value, tasks = fib_value_and_tasks(n)
            for i in range(a.launches):
                res, st = gt.launch([gt.fib_root(n)])
                if res[0].status != gt.ROOT_DONE or res[0].value != value or res[0].tasks != tasks:
                    print("fib30 launch %d: wrong result" % i, file=sys.stderr)
                    return 1
                print("fib30 launch %d: %.3f ms, %d tasks, %d executions" % (i, st.kernel_ms, res[0].tasks,
                                                                            int(st.counters[1])), flush=True)
            return 0
        src = torch.from_numpy(gt.gen_keys(42, n)).cuda()
        arr = torch.empty_like(src)
        tmp = torch.empty_like(src)
        want = torch.sort(src).values
        if a.case == "mergesort":
            root = gt.mergesort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 128, 256)
        else:
            root = gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 2048, 2048)
        for i in range(a.launches):
            res, st = gt.launch([root])
            if res[0].status != gt.ROOT_DONE or not torch.equal(arr, want):
                print("%s launch %d: wrong output (status %d)" % (a.case, i, res[0].status), file=sys.stderr)
                return 1
            print("%s launch %d: %.3f ms, %d tasks, %d executions" % (a.case, i, st.kernel_ms, res[0].tasks,
                                                                     int(st.counters[1])), flush=True)
    finally:
        gt.gtap_finalize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
