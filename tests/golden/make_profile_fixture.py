"""Writes tests/golden/profile/: the profiler CSVs of one small fib run on a
GPU (fib(18) on 2 blocks of 64 threads, 256 timeline samples per warp), as
gtap_visualize_profile writes them in the reference's layout.  The CPU test
tests/test_visualizer_cpu.py reads them with the reference's visualiser.

    python tests/golden/make_profile_fixture.py      (needs a B200)
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main():
    import torch
    import gtap_b200 as gt
    from tests import oracle_lib as orc
    torch.cuda.init()
    out = os.path.join(HERE, "profile")
    os.makedirs(out, exist_ok=True)
    gt.gtap_initialize(gt.default_config(grid=2, block=64, profile_samples=256))
    try:
        res, st = gt.launch([gt.fib_root(18)])
        assert res[0].value == orc.fib(18) and st.status == 0
        gt.gtap_visualize_profile("fib", out)
    finally:
        gt.gtap_finalize()
    print(sorted(os.listdir(out)))


if __name__ == "__main__":
    main()
