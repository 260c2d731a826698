"""Autotuner for the scheduler's launch parameters.

The reference fixes its scheduler geometry at compile time (GTAP_BLOCK_SIZE,
GRID, GTAP_MAX_TASKS_PER_WARP, GTAP_NUM_QUEUES in
runtime/detail/common/gtap_config.cuh:6-28); here they are launch-time fields
of gtap_config, so they can be searched per workload and device.

Search: coordinate descent from the library defaults over
  block          threads per block (warps per block = block / 32)
  warps_per_sm   resident workers per SM (grid = warps_per_sm * SMs / warps per block,
                 capped by the kernel's occupancy)
  deque_capacity per worker and queue
  steal_batch    tasks moved by one steal
  probe_width    victims probed in parallel per steal attempt
  victim_policy  random / last success / fullest of the probed
  num_queues     EPAQ queues
  spawn_capacity children staged per worker and round (shared memory per warp,
                 so it also sets how many workers fit an SM)
  leaf_batch     sort and merge leaves a warp stages in shared memory at once
                 (one load round trip per batch, 1 KB of shared memory each)
  publish_lazy   0: publish every ready task beyond the next batch each round;
                 1: keep up to a batch in reserve privately until some worker is
                 idle (fuller rounds once the GPU is busy, a slower ramp-up);
                 2: 1 without sort leaves, 0 in the sorting kernel
  join_walk      rounds of at most this many tasks run fib's sums at their joins
                 (0: never); the tree's drain gains, full rounds would wait
  sub_rounds     extra passes of task bodies on a round's idle lanes over the
                 children the round staged (fib / n-queens launches)
  max_inflight_roots  roots admitted and not finished, at most (0: no limit);
                 an asynchronous BFS relaxes vertices more than once the more
                 roots share the GPU, so served batches of BFS roots do less
                 work with fewer of them in flight
Each trial re-initialises the runtime with the candidate configuration, runs
one warm-up launch and `reps` timed launches (CUDA events around the
persistent kernel) and keeps the median.  Every trial's results must equal the
first trial's (values, task counts of deterministic kinds, statuses), so a
configuration that breaks a result cannot win.

    python -m gtap_b200.autotune --workload mix --out gtap_b200/tuned/b200_mix.json
    python -m gtap_b200.autotune --workload serve --out gtap_b200/tuned/b200_serve.json
    python -m gtap_b200.autotune --workload cilksort26_block --out gtap_b200/tuned/b200_cilksort26_block.json
    python -m gtap_b200.autotune --workload mergesort24 --out gtap_b200/tuned/b200_mergesort24.json

The serve workload is the served roots (BFS on R-MAT 16-20, tree sums of
2^18-2^20 nodes, 200 of them) in one batch launch of the kernel serve mode
runs, the session's capacity when every root arrives at once, admitted in
arrival order as a session admits them; BFS depth arrays are reset before
every launch, and a BFS root's task count (timing-dependent) is left out of
the result check.
"""
import argparse
import json
import os
import statistics
import sys
import time

SPACE = {
    "warps_per_sm": [4, 8, 12, 16, 24, 32],
    "block": [32, 64, 128, 256, 512, 1024],
    "deque_capacity": [256, 1024, 4096, 8192],
    "steal_batch": [1, 8, 32],
    "probe_width": [1, 4, 16, 32],
    "victim_policy": [0, 1, 2],
    "num_queues": [1, 2, 4],
    "spawn_capacity": [128, 256, 512, 1024],
    "max_inflight_roots": [0, 8, 16, 32, 64, 128],
    "publish_lazy": [0, 1, 2],
    "leaf_batch": [1, 2, 4],
    "join_walk": [0, 2, 4, 8, 32],
    "sub_rounds": [0, 1, 2, 4, 8],
}
ORDER = ["publish_lazy", "max_inflight_roots", "leaf_batch", "warps_per_sm", "block", "steal_batch", "deque_capacity", "probe_width",
         "victim_policy", "num_queues", "spawn_capacity", "join_walk", "sub_rounds"]


def to_overrides(point, sm_count):
    """Tuner point -> gtap_config field overrides."""
    o = {k: v for k, v in point.items() if k != "warps_per_sm"}
    block = point.get("block", 256)
    wpb = max(1, block // 32)
    if "warps_per_sm" in point:
        o["grid"] = max(1, (point["warps_per_sm"] * sm_count) // wpb)
    return o


def coordinate_descent(measure, start, space=SPACE, order=ORDER, sweeps=2, log=None):
    """Minimise measure(point) -> seconds (or None when the point is invalid)
    one coordinate at a time.  Returns (best_point, best_time, trials)."""
    best = dict(start)
    cache = {}

    def evaluate(p):
        key = tuple(sorted(p.items()))
        if key not in cache:
            cache[key] = measure(p)
            if log:
                log(p, cache[key])
        return cache[key]

    best_t = evaluate(best)
    if best_t is None:
        raise ValueError("the starting point is not valid")
    for _ in range(sweeps):
        improved = False
        for name in order:
            for v in space[name]:
                if v == best.get(name):
                    continue
                cand = dict(best)
                cand[name] = v
                t = evaluate(cand)
                if t is not None and t < best_t:
                    best, best_t, improved = cand, t, True
        if not improved:
            break
    trials = [{"point": dict(k), "s": v} for k, v in cache.items()]
    return best, best_t, trials


def _signature(gt, res, kinds=None):
    """What must not change between configurations: status, value and task
    count of every root, except the task count of an asynchronous BFS (one
    task per successful relaxation, which depends on timing)."""
    out = []
    for i, r in enumerate(res):
        bfs = kinds is not None and kinds[i] == gt.KIND_BFS
        out.append((r.status, r.value, None if bfs else r.tasks))
    return out


def run(workload="mix", reps=3, sweeps=2, n_roots=None, out=None, quiet=False, start_point=None):
    import torch
    import gtap_b200 as gt
    from gtap_b200 import workloads as wl

    torch.cuda.init()
    sm_count = torch.cuda.get_device_properties(0).multi_processor_count
    keep = []
    before = None   # runs before every launch (resets what a launch consumes)
    check = None    # checks the warm-up launch's output beyond values and task counts
    fixed = {}      # overrides every trial carries
    space, order = SPACE, ORDER
    if workload == "mix":
        mix = wl.Mix(gt, n_roots or wl.N_ROOTS)
        src, arr, tmp = mix.device_slabs()
        keep += [src, arr, tmp]
        roots = mix.roots(gt, src.data_ptr(), arr.data_ptr(), tmp.data_ptr())
    elif workload == "serve":
        # the served workload's roots (BFS on R-MAT 16-20, tree sums of
        # 2^18-2^20 nodes) in one batch launch of the kernel serve mode runs:
        # the session's capacity when every root is enqueued at once
        from gtap_b200.serve_bench import ServeWorkload
        sw = ServeWorkload(gt)
        roots, depths = sw.roots(sw.draw(n_roots or 200))
        keep += [sw, depths]
        fixed["admit_order"] = gt.ADMIT_AS_GIVEN

        def before():
            for d in depths:
                if d is not None:
                    d.fill_(0x3f3f3f3f)
    elif workload == "cilksort26_block":
        # block-cooperative cilksort of 2^26 mt19937(42) keys, cutoffs
        # 2048/2048; one worker per block, so warps per SM reach 64 and only
        # the axes the block scheduler reads are searched
        n = n_roots or (1 << 26)
        src = torch.from_numpy(gt.gen_keys(42, n)).cuda()
        arr = torch.empty_like(src)
        tmp = torch.empty_like(src)
        want = torch.sort(src).values
        keep += [src, arr, tmp, want]
        roots = [gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 2048, 2048)]
        fixed["mode"] = gt.MODE_BLOCK
        space = dict(SPACE, warps_per_sm=[16, 32, 48, 64], block=[64, 128, 256, 512])
        order = ["warps_per_sm", "block", "deque_capacity", "probe_width", "victim_policy"]

        def check():
            return bool(torch.equal(arr, want))
    elif workload == "mergesort24":
        # thread-mode mergesort of 2^24 mt19937(42) keys, cutoff 128 and merge
        # cutoff 256 (examples/mergesort/mergesort.cu's settings)
        n = n_roots or (1 << 24)
        src = torch.from_numpy(gt.gen_keys(42, n)).cuda()
        arr = torch.empty_like(src)
        tmp = torch.empty_like(src)
        want = torch.sort(src).values
        keep += [src, arr, tmp, want]
        roots = [gt.mergesort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 128, 256)]
        order = ["warps_per_sm", "block", "leaf_batch", "spawn_capacity", "steal_batch", "deque_capacity",
                 "probe_width", "victim_policy", "publish_lazy"]

        def check():
            return bool(torch.equal(arr, want))
    else:
        roots = wl.single_root_workload(gt, workload)
    kinds = [r.kind for r in roots]
    # every kind in these workloads has a fixed task tree (cilksort's depends
    # only on the keys), so values and task counts must not change
    ref_sig = {}

    def measure(point):
        over = to_overrides(point, sm_count)
        over.update(fixed)
        try:
            gt.gtap_initialize(gt.default_config(**over))
        except gt.GtapError:
            return None
        try:
            if before:
                before()
            res, st = gt.launch(roots)                      # warm-up
            if check is not None and not check():
                raise RuntimeError("configuration %s gave a wrong output" % over)
            sig = _signature(gt, res, kinds)
            if "sig" not in ref_sig:
                ref_sig["sig"] = sig
            elif sig != ref_sig["sig"]:
                raise RuntimeError("configuration %s changed a result" % over)
            ms = []
            for _ in range(reps):
                if before:
                    before()
                res, st = gt.launch(roots)
                ms.append(st.kernel_ms)
            return statistics.median(ms) / 1e3
        except gt.GtapError:
            return None
        finally:
            gt.gtap_finalize()

    def log(p, t):
        if not quiet:
            print("%-110s %s" % (json.dumps(p), "invalid" if t is None else "%.3f ms" % (t * 1e3)), flush=True)

    defaults = gt.default_config()
    start = {"warps_per_sm": 8, "block": defaults.block, "deque_capacity": defaults.deque_capacity,
             "steal_batch": defaults.steal_batch, "probe_width": defaults.probe_width,
             "victim_policy": defaults.victim_policy, "num_queues": defaults.num_queues,
             "spawn_capacity": defaults.spawn_capacity, "max_inflight_roots": defaults.max_inflight_roots,
             "publish_lazy": defaults.publish_lazy, "leaf_batch": defaults.leaf_batch,
             "join_walk": defaults.join_walk, "sub_rounds": defaults.sub_rounds}
    if workload == "cilksort26_block":
        start = {"warps_per_sm": 64, "block": defaults.block, "deque_capacity": defaults.deque_capacity,
                 "probe_width": defaults.probe_width, "victim_policy": defaults.victim_policy}
    start.update(start_point or {})
    t0 = time.time()
    best, best_t, trials = coordinate_descent(measure, start, space=space, order=order, sweeps=sweeps, log=log)
    best_over = to_overrides(best, sm_count)
    best_over.update(fixed)
    result = {"workload": workload, "roots": len(roots), "device": torch.cuda.get_device_name(0),
              "sm_count": sm_count, "best_point": best, "best_overrides": best_over,
              "best_kernel_ms": best_t * 1e3, "reps": reps, "trials": len(trials),
              "search_s": time.time() - t0,
              "table": sorted(({"point": t["point"], "kernel_ms": None if t["s"] is None else t["s"] * 1e3}
                               for t in trials), key=lambda e: (e["kernel_ms"] is None, e["kernel_ms"] or 0))}
    if out:
        os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
        with open(out, "w") as f:
            json.dump(result, f, indent=1)
    return result


def load_tuned(path):
    """gtap_config overrides from a tuner result file, or {} if absent."""
    try:
        with open(path) as f:
            return dict(json.load(f)["best_overrides"])
    except (OSError, KeyError, ValueError):
        return {}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", default="mix",
                    choices=["mix", "serve", "fib30", "fib34c12", "nq13", "nq13c7", "cilksort26_block", "mergesort24"])
    ap.add_argument("--roots", type=int, default=None)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--out", default=None)
    ap.add_argument("--start", default="", help="json point to start the descent from (keys of the search space)")
    a = ap.parse_args(argv)
    r = run(a.workload, a.reps, a.sweeps, a.roots, a.out, start_point=json.loads(a.start) if a.start else None)
    print(json.dumps({k: r[k] for k in ("workload", "best_point", "best_overrides", "best_kernel_ms", "trials")}))


if __name__ == "__main__":
    sys.exit(main())
