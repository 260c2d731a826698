#!/usr/bin/env python
"""Benchmark of the B200 GTaP runtime on the batched 4096-root mix.

Workload (one step): 4096 independent fork-join roots from the seeded mix
(gtap_gen_mix(42, 4096): fib(n in [18,28]) cutoff 0, n-queens(n in [8,11])
one task per row, cilksort of mt19937 int32 keys with sizes in [2^10, 2^20)
and cutoffs 64/256) in one batch call (gtap_launch): admitted grouped by kind
and run as two persistent launches, the fib and n-queens roots and then the
cilksort roots.  Metric: tasks/s (spawned tasks, root included).  Inputs are
resident in HBM when the timed region starts; the key slabs (~2.6 GB) exceed
L2, and each step's cilksort leaves read the pristine input, so no restore
happens between steps.

Prints ONE JSON line (rank 0).  --impl reference times the reference's
sequential programs (CPU, the oracle's restatement of seq_fib.c / seq_nq.c /
seq_cilksort.cpp) on a bounded sample of the same roots; it builds the mix
with the oracle's own generators and never loads libgtap_b200.so.  Both arms
print the same `config` object.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# plain-Python modules of the package: importing them loads no library
from gtap_b200.workloads import MERGE_CUTOFF, MIX_SEED, N_ROOTS, SORT_CUTOFF, Mix  # noqa: E402
from gtap_b200.autotune import load_tuned  # noqa: E402

METRIC = "tasks_per_sec_batched_4096_root_mix"
UNIT = "tasks/s"
TUNED = os.path.join(ROOT, "gtap_b200", "tuned", "b200_mix.json")
BLOCK_TUNED = os.path.join(ROOT, "gtap_b200", "tuned", "b200_cilksort26_block.json")
MSORT_TUNED = os.path.join(ROOT, "gtap_b200", "tuned", "b200_mergesort24.json")

# algorithmic bytes per task (frame S written by the parent + read by the child,
# 8 B deque slot, 8 B join RMW, 4 B result), frame sizes of the lowered tasks
S_FIB, S_NQ, S_SORT, S_MERGE = 16, 16, 28, 32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--roots", type=int, default=N_ROOTS)
    ap.add_argument("--cpu-sample-s", type=float, default=15.0, help="target seconds of CPU baseline work")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-per-root", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--block-keys", type=int, default=1 << 26,
                    help="keys of the block-mode cilksort run (cutoffs 2048/2048); 0 = no block run")
    ap.add_argument("--mergesort-keys", type=int, default=1 << 24,
                    help="keys of the thread-mode mergesort run (cutoff 128); 0 = no mergesort run")
    ap.add_argument("--serve-roots", type=int, default=200,
                    help="roots per serve session (BFS on R-MAT 16-20 / tree sums 2^18-2^20); 0 = no serve run")
    ap.add_argument("--config", default="", help="json dict of gtap_config overrides (applied last)")
    ap.add_argument("--tuned", default=TUNED, help="autotuner result whose overrides are applied first ('' = none)")
    ap.add_argument("--no-reference-gpu", dest="reference_gpu", action="store_false",
                    help="skip the fib comparison with the reference GTaP GPU build")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the reference's published configurations and the single-root BFS / tree runs")
    return ap.parse_args()


def algorithmic_bytes(mix, results):
    """Bytes per step the algorithm must move, as (fib and n-queens roots,
    cilksort roots).  fib tasks: the parent's argument write and the child's
    read of a frame, the deque slot write and read, the join-counter update and
    the result read.  n-queens tasks (no join): the frame write and read and
    the deque slot.  cilksort roots: each task's frame, deque slot and join
    counter, plus 8 bytes per key (a 4-byte read and write) for the leaf pass
    and for two merge passes per four-way level."""
    light = sort = 0
    for i, r in enumerate(results):
        k = int(mix.kind[i])
        if k == 0:
            light += r.tasks * (2 * S_FIB + 8 + 8 + 4)
        elif k == 1:
            light += r.tasks * (2 * S_NQ + 8)
        else:
            n = int(mix.param[i])
            levels, m = 0, n
            while m >= SORT_CUTOFF:
                m //= 4
                levels += 1
            sort += r.tasks * (2 * S_MERGE + 8 + 8)     # task overhead
            sort += n * 8 * (1 + 2 * levels)             # leaf pass + two merge passes per level
    return light, sort


# the mix's first launch holds only fib and n-queens roots, so the runtime picks
# the kernel with those two bodies (BuiltinProgramLight adds BFS and tree sums)
LIGHT_KERNEL = "gtap::thread_worker_kernel_lb<BuiltinProgramFibNq>"
FULL_KERNEL = "gtap::thread_worker_kernel<BuiltinProgram>"


def worker_kernels(alg_light, alg_sort, light_ms, full_ms, hbm):
    """Per worker kernel of a step: its roots, mean launch time, algorithmic
    bytes and the fraction of the measured copy bandwidth they come to.  A
    split batch runs the fib and n-queens roots in the kernel without sort
    leaves and the cilksort roots in the sort-capable one; an unsplit batch
    runs all of them in the sort-capable kernel."""
    out = []
    if light_ms > 0:
        out.append({"kernel": LIGHT_KERNEL, "roots": "fib and n-queens", "ms": light_ms,
                    "algorithmic_bytes": alg_light, "traffic": scaled_traffic("light_kernel", alg_light)})
        if full_ms > 0:
            out.append({"kernel": FULL_KERNEL, "roots": "cilksort", "ms": full_ms, "algorithmic_bytes": alg_sort,
                        "traffic": scaled_traffic("sort_kernel", alg_sort)})
    else:
        out.append({"kernel": FULL_KERNEL, "roots": "all", "ms": full_ms, "algorithmic_bytes": alg_light + alg_sort,
                    "traffic": scaled_traffic("mixed_kernel", alg_light + alg_sort)})
    for k in out:
        k["achieved_gbs"] = k["algorithmic_bytes"] / (k["ms"] / 1e3) / 1e9
        k["frac"] = k["achieved_gbs"] / hbm
    return out


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        return self.summarize(self.lines)

    @staticmethod
    def summarize(lines):
        """Median SM clock, the max clock and the throttle reasons active in any
        sample, from `nvidia-smi --query-gpu=<Q> --format=csv,noheader,nounits` lines."""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's sequential recursions on a bounded sample
# ---------------------------------------------------------------------------
class OracleGenerators:
    """The oracle's restatement of the seeded generators (std::mt19937_64 root
    mix, std::mt19937 keys).  The reference arm builds the mix with these, so
    it never loads the product library."""

    def __init__(self):
        from tests import oracle_lib as orc
        self.orc = orc

    def gen_mix(self, seed, n):
        return self.orc.root_mix(seed, n)

    def gen_keys(self, seed, n):
        return self.orc.keys(seed, n)


def workload_config(mix):
    """The `config` object both arms print (identical by construction)."""
    return {"workload": "batched 4096-root mix: fib(n in [18,28], cutoff 0), n-queens(n in [8,11], one task per "
                        "row), cilksort of 2^10..2^20 std::mt19937 int32 keys (cutoffs 64/256)",
            "roots": int(mix.n), "mix_seed": MIX_SEED, "cilksort_keys": int(mix.total_keys),
            "l2": "inputs larger than L2 (%.2f GB of key slabs: source, output, scratch)"
                  % (3 * mix.total_keys * 4 / 1e9)}


def cpu_sample(mix, target_s, cores):
    """Roots (seeded order) whose summed single-core time estimate reaches
    target_s * cores.  The cost model only sizes the sample."""
    nq_nodes = {8: 2057, 9: 8394, 10: 35539, 11: 166926}   # search-tree nodes of n-queens(n)
    est = {0: lambda p: 1.6e-9 * 1.618 ** p, 1: lambda p: 1.2e-8 * nq_nodes.get(p, 6.0 ** p),
           2: lambda p: 9e-8 * p}
    budget = target_s * cores
    order = np.random.RandomState(7).permutation(mix.n)
    picked, spent = [], 0.0
    for i in order:
        c = est[int(mix.kind[i])](int(mix.param[i]))
        if spent + c > budget and picked:
            continue
        picked.append(int(i))
        spent += c
        if spent >= budget:
            break
    return picked


def cpu_baseline(mix, sample, tasks_of, cores, steps=1):
    """The sample's roots on `cores` host threads (each a C call that releases
    the GIL): fib / n-queens as the sequential recursions of seq_fib.c /
    seq_nq.c, cilksort as seq_cilksort.cpp's recursion on a fresh copy of the
    root's keys.  Keys are copied before the timed region; each step's wall
    time covers only the recursions.  Returns one tasks/s figure per step."""
    from concurrent.futures import ThreadPoolExecutor
    from tests import oracle_lib as orc
    L = orc.load()
    tasks = int(sum(int(tasks_of(i)) for i in sample))
    # largest jobs first: the makespan is not set by a big root started last
    sample = sorted(sample, key=lambda i: -(int(mix.param[i]) * (50 if mix.kind[i] == 2 else 1)))
    values, walls = [], []
    with ThreadPoolExecutor(cores) as pool:
        for _ in range(steps):
            bufs = {}
            for i in sample:
                if int(mix.kind[i]) == 2:
                    o, n = int(mix.offsets[i]), int(mix.param[i])
                    bufs[i] = (mix.keys[o:o + n].copy(), np.empty(n, np.int32))

            def job(i):
                k = int(mix.kind[i])
                if k == 2:
                    a, t = bufs[i]
                    L.orc_seq_cilksort(orc.p(a), orc.p(t), len(a))
                else:
                    L.orc_seq_root(k, int(mix.param[i]), int(mix.seed[i]))

            t0 = time.perf_counter()
            list(pool.map(job, sample))
            wall = time.perf_counter() - t0
            for a, _ in bufs.values():
                assert np.all(a[1:] >= a[:-1])
            values.append(tasks / wall)
            walls.append(wall)
    return values, walls, tasks


def mix_tasks_oracle(mix, sample):
    """Per-root task counts of the sampled roots: fib / n-queens from the
    recursions' closed counts, cilksort by running the oracle's cilksort
    recursion on the root's keys (its merge splits depend on them)."""
    from tests import oracle_lib as orc
    out = {}
    for i in sample:
        k, p = int(mix.kind[i]), int(mix.param[i])
        if k == 0:
            out[i] = orc.fib_tasks(p, 0)
        elif k == 1:
            out[i] = orc.nq_tasks(p, p - 1)
        else:
            o = int(mix.offsets[i])
            _, st, mt = orc.cilksort(mix.keys[o:o + p], SORT_CUTOFF, MERGE_CUTOFF)
            out[i] = st + mt
    return out


# ---------------------------------------------------------------------------
def run_reference(args, rank):
    if rank != 0:
        return
    mix = Mix(OracleGenerators(), args.roots)
    cores = os.cpu_count() or 1
    sample = cpu_sample(mix, max(2.0, args.cpu_sample_s / max(1, args.steps)), cores)
    tpr = mix_tasks_oracle(mix, sample)
    _, _, _ = cpu_baseline(mix, sample, tpr.get, cores, steps=max(1, args.warmup))   # warm-up steps
    values, walls, tasks = cpu_baseline(mix, sample, tpr.get, cores, steps=args.steps)
    v = statistics.median(values)
    cb = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
          "sample": "%d of %d mix roots per step (%d tasks): the oracle's restatement of seq_fib.c / seq_nq.c / "
                    "seq_cilksort.cpp, -O2, one root per host thread" % (len(sample), mix.n, tasks)}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(walls) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded mix, mt19937 keys)", "config": workload_config(mix),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    import gtap_b200 as gt

    overrides = load_tuned(args.tuned) if args.tuned else {}
    tuned_from = os.path.relpath(args.tuned, ROOT) if overrides else None
    overrides.update(json.loads(args.config) if args.config else {})
    cfg = gt.gtap_initialize(gt.default_config(**overrides))
    mix = Mix(gt, args.roots)
    src = torch.from_numpy(mix.keys).cuda()
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    roots = mix.roots(gt, src.data_ptr(), arr.data_ptr(), tmp.data_ptr())

    # warm-up (the first launch's results are verified)
    res, verified = None, False
    for w in range(max(1, args.warmup)):
        res, st = gt.launch(roots)
        if w == 0:
            verified = verify(gt, mix, res, src, arr)

    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kern_ms, tasks_step, stats_acc = [], [], None
    e0.record()
    light_ms = []
    for _ in range(args.steps):
        res, st = gt.launch(roots)
        kern_ms.append(st.kernel_ms)
        light_ms.append(st.light_kernel_ms)
        tasks_step.append(sum(r.tasks for r in res))
        stats_acc = st
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ck = clocks.stop()
    ms_max = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    tasks_per_step = int(statistics.median(tasks_step))
    value = world * tasks_per_step * args.steps / (ms_max / 1e3)
    # the last timed launch's results must be the verified ones
    verified = verified and all(r.status == gt.ROOT_DONE for r in res) and tasks_per_step == tasks_step[0]

    # roofline: the dominant kernel = the worker kernel with the larger share of the step
    alg_light, alg_sort = algorithmic_bytes(mix, res)
    k_ms = statistics.mean(kern_ms)
    l_ms = statistics.mean(light_ms)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    kernels = worker_kernels(alg_light, alg_sort, l_ms, k_ms - l_ms, hbm)
    top = max(kernels, key=lambda k: k["ms"])
    counters = stats_acc.as_dict() if stats_acc else {}
    roof = {"bound": "hbm", "achieved": top["achieved_gbs"], "peak": hbm, "unit": "GB/s", "frac": top["frac"],
            "traffic": top["traffic"], "peak_source": peak_src, "kernel": top["kernel"], "kernel_ms": top["ms"],
            "algorithmic_bytes_per_launch": top["algorithmic_bytes"], "worker_kernels": kernels,
            "worker_ms_per_step": k_ms, "atomic": atomic_view(counters, mix, res, k_ms)}

    # e2e through the host-buffer entry point (H2D keys, D2H sorted keys + results)
    e2e = None
    if not args.no_e2e:
        e2e = measure_e2e(gt, mix, args.steps, tasks_per_step, world, arr)

    # per-root launch baseline (gtap_reset-style relaunch per root), 1 step,
    # under its own best configuration among the library defaults and the
    # batch-tuned one
    per_root = None
    if not args.no_per_root:
        per_root = measure_per_root(gt, roots, res, value / world, overrides)

    # serve mode: capacity, then Poisson arrivals at fractions of it and at
    # 2000, 5000 and 10000 roots/s (the low end of the served rates asked
    # for), with the configuration
    # the autotuner found for the served roots (library defaults without one)
    serve = None
    if args.serve_roots > 0:
        gt.gtap_finalize()
        from gtap_b200 import serve_bench
        serve_tuned = os.path.join(ROOT, "gtap_b200", "tuned", "b200_serve.json")
        serve_cfg = load_tuned(serve_tuned)
        sv = serve_bench.run(loads=(0.5, 0.9), rates=(2000, 5000, 10000), count=args.serve_roots, config=serve_cfg)
        keys = ("load", "rate_roots_per_s", "throughput_roots_per_s", "tasks_per_s", "latency_ms",
                "device_service_ms", "ok")
        serve = {"workload": "50% async BFS on R-MAT scale 16-20 (edge factor 16), 50% int64 tree sums over "
                             "2^18-2^20-node unbalanced binary trees; Poisson arrivals",
                 "roots_per_session": args.serve_roots,
                 "config": os.path.relpath(serve_tuned, ROOT) if serve_cfg else "library defaults",
                 "capacity_roots_per_s": sv["capacity"]["throughput_roots_per_s"],
                 "capacity_tasks_per_s": sv["capacity"]["tasks_per_s"],
                 "sessions": [{k: r[k] for k in keys} for r in [sv["capacity"]] + sv["sessions"]],
                 "ok": sv["capacity"]["ok"] and all(r["ok"] for r in sv["sessions"])}

    # block-cooperative mode: cilksort of mt19937(42) keys, cutoffs 2048/2048
    block = None
    if args.block_keys > 0:
        gt.gtap_finalize()
        block = measure_block_cilksort(gt, args.block_keys, args.steps, args.warmup,
                                       cpu=not args.no_cpu and rank == 0 and world == 1, hbm_peak=hbm,
                                       overrides=json.loads(args.config) if args.config else {},
                                       tuned=BLOCK_TUNED if args.tuned else "")

    # thread mode: mergesort of mt19937(42) keys (examples/mergesort/mergesort.cu's cutoff 128)
    msort = None
    if args.mergesort_keys > 0:
        gt.gtap_finalize()
        msort = measure_mergesort_thread(gt, args.mergesort_keys, args.steps, args.warmup, hbm_peak=hbm,
                                         overrides=json.loads(args.config) if args.config else {},
                                         tuned=MSORT_TUNED if args.tuned else "")

    # the reference GTaP GPU build on fib, beside this runtime (same box, same call),
    # and as the per-root baseline for the mix's fib roots
    ref_gpu = None
    if args.reference_gpu and rank == 0:
        gt.gtap_finalize()
        ref_gpu = measure_reference_gpu(gt)
        ref_gpu["per_root_fib_roots_of_the_mix"] = measure_reference_per_root(gt, mix, overrides)

    published = single = None
    if args.extras and rank == 0:
        gt.gtap_finalize()
        published = measure_published_configs(gt)
        single = measure_single_roots(gt)

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        tasks_gpu = [r.tasks for r in res]
        cores = os.cpu_count() or 1
        sample = cpu_sample(mix, args.cpu_sample_s, cores)
        vals, walls, ntasks = cpu_baseline(mix, sample, lambda i: tasks_gpu[i], cores)
        cpu = {"value": vals[0], "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "%d of %d mix roots (%d tasks), %.1f s wall: the oracle's restatement of seq_fib.c / "
                         "seq_nq.c / seq_cilksort.cpp, -O2, one root per host thread"
                         % (len(sample), mix.n, ntasks, walls[0])}

    W = int(counters.get("workers", 0))
    sched = {"steal_success_rate": counters.get("steal_successes", 0) / max(1, counters.get("steal_attempts", 0)),
             "idle_worker_fraction": counters.get("idle_ns", 0) / max(1.0, stats_acc.worker_ms() * 1e6),
             "workers": W, "light_workers": int(counters.get("light_workers", 0)),
             "launches_per_step": int(counters.get("launches", 1)), "idle_polls": counters.get("idle_polls", 0),
             "executions": counters.get("executions", 0), "rounds": counters.get("rounds", 0),
             "tasks_per_round": counters.get("executions", 0) / max(1, counters.get("rounds", 0))}
    # order: the contract's keys first, the large per-mode objects next, the
    # short summaries last (they stay in view when the line is cut short)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded mix, mt19937 keys)",
            "config": workload_config(mix), "tasks_per_step": tasks_per_step,
            "parallelism": "replicas" if world > 1 else "single GPU",
            "runtime": {"config": cfg.as_dict(), "tuned_from": tuned_from},
            "verified": verified, "gpu_launches": 2 * int(counters.get("launches", 1)) * args.steps, "e2e": e2e, "roofline": roof,
            "cpu_baseline": cpu, "clocks": ck, "serve": serve, "block_mode": block, "mergesort_thread": msort,
            "single_roots": single, "published_configs": published,
            "reference_gpu": ref_gpu, "per_root_launch": per_root, "scheduler": sched}
    if rank == 0:
        print(json.dumps(line), flush=True)
    gt.gtap_finalize()
    if world > 1:
        dist.destroy_process_group()


def max_over_ranks(x, world, device):
    """The largest of every rank's x (the job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cilksort_bytes(n, sort_cutoff):
    """Algorithmic HBM bytes of cilksort(n): a leaf reads its keys and writes
    them sorted (8 B/key); an inner node's three merges read and write every
    key twice (16 B/key) on top of its four quarters."""
    if n < sort_cutoff:
        return 8 * n
    h = n // 2
    q1, q3 = h // 2, (n - h) // 2
    return 16 * n + sum(cilksort_bytes(m, sort_cutoff) for m in (q1, h - q1, q3, n - h - q3))


def mergesort_bytes(n, cutoff):
    """Algorithmic HBM bytes of mergesort(n): a leaf reads its keys and writes
    them sorted, every merge reads and writes the keys of its node (8 B/key)."""
    if n <= cutoff or n <= 1:
        return 8 * n
    nl = (n + 1) // 2
    return 8 * n + mergesort_bytes(nl, cutoff) + mergesort_bytes(n - nl, cutoff)


def measure_mergesort_thread(gt, n, steps, warmup, hbm_peak, overrides=None, tuned=""):
    """mergesort of n keys (std::mt19937(42)) in thread mode, cutoff 128 and
    merge cutoff 256, one root per launch with the tuner's result `tuned`
    (library defaults without one) plus explicit overrides; checked against a
    plain sort."""
    import torch
    keys = gt.gen_keys(42, n)
    src = torch.from_numpy(keys).cuda()
    out = torch.empty_like(src)
    tmp = torch.empty_like(src)
    over = load_tuned(tuned) if tuned else {}
    over.update(overrides or {})
    gt.gtap_initialize(gt.default_config(**over))
    root = gt.mergesort_root(src.data_ptr(), out.data_ptr(), tmp.data_ptr(), n, 128, 256)
    for _ in range(max(1, warmup)):
        res, st = gt.launch([root])
    ok = bool(np.array_equal(out.cpu().numpy(), np.sort(keys))) and st.status == 0
    ms = []
    for _ in range(steps):
        res, st = gt.launch([root])
        ms.append(st.kernel_ms)
    gt.gtap_finalize()
    k_ms = statistics.mean(ms)
    alg = mergesort_bytes(n, 128)
    achieved = alg / (k_ms / 1e3) / 1e9
    ratio = traffic_from_profile("mergesort_kernel_traffic_over_algorithmic")
    return {"workload": "mergesort of %d int32 keys (std::mt19937(42)), thread mode, cutoff 128, merge cutoff 256, "
                        "one root per launch" % n,
            "keys": n, "ms_per_sort": k_ms, "keys_per_s": n / (k_ms / 1e3), "tasks": res[0].tasks,
            "tasks_per_s": res[0].tasks / (k_ms / 1e3), "sorted_equals_plain_sort": ok,
            "config": os.path.relpath(tuned, ROOT) if tuned and load_tuned(tuned) else "library defaults",
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "algorithmic_bytes_per_launch": alg,
                         "traffic": None if ratio is None else int(alg * ratio),
                         "kernel": "gtap::thread_worker_kernel<BuiltinProgram>"}}


def measure_block_cilksort(gt, n, steps, warmup, cpu, hbm_peak, overrides=None, tuned=""):
    """cilksort of n keys (std::mt19937(42), full int32 range) in block mode,
    one root per launch, inputs resident; leaves read the pristine input so
    no restore is needed between launches.  Checked against a plain sort.
    The configuration: the block-mode tuner result `tuned` (library defaults
    without one), then the explicit overrides."""
    import torch
    keys = gt.gen_keys(42, n)
    src = torch.from_numpy(keys).cuda()
    arr = torch.empty_like(src)
    tmp = torch.empty_like(src)
    over = load_tuned(tuned) if tuned else {}
    over.update(overrides or {})
    over["mode"] = gt.MODE_BLOCK
    gt.gtap_initialize(gt.default_config(**over))
    root = gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 2048, 2048)
    for _ in range(max(1, warmup)):
        res, st = gt.launch([root])
    want = np.sort(keys)
    ok = bool(np.array_equal(arr.cpu().numpy(), want)) and st.status == 0
    ms = []
    for _ in range(steps):
        res, st = gt.launch([root])
        ms.append(st.kernel_ms)
    k_ms = statistics.mean(ms)
    tasks = res[0].tasks
    alg = cilksort_bytes(n, 2048)
    achieved = alg / (k_ms / 1e3) / 1e9
    out = {"workload": "cilksort of %d int32 keys (std::mt19937(42)), block-cooperative mode, sort and merge "
                       "cutoffs 2048, one root per launch" % n,
           "keys": n, "ms_per_sort": k_ms, "keys_per_s": n / (k_ms / 1e3), "tasks": tasks,
           "tasks_per_s": tasks / (k_ms / 1e3), "grid": st.grid, "block": st.block,
           "config": os.path.relpath(tuned, ROOT) if tuned and load_tuned(tuned) else "library defaults",
           "executions": int(st.counters[1]), "join_finishes": int(st.counters[10]),
           "steal_success_rate": int(st.counters[4]) / max(1, int(st.counters[3])),
           "sorted_equals_plain_sort": ok,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                        "frac": achieved / hbm_peak, "algorithmic_bytes_per_launch": alg,
                        "traffic": (None if traffic_from_profile("block_kernel_traffic_over_algorithmic") is None
                                    else int(alg * traffic_from_profile("block_kernel_traffic_over_algorithmic"))),
                        "kernel": "gtap::block_worker_kernel<BlockProgram>"}}
    gt.gtap_finalize()
    if cpu:
        sys.path.insert(0, ROOT)
        from tests import oracle_lib as orc   # the CPU leg: std::sort of the same keys, one core
        k2 = keys.copy()
        t0 = time.perf_counter()
        orc.load().orc_sort_i32(orc.p(k2), len(k2))
        wall = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n / wall, "unit": "keys/s", "cores": 1, "kind": "port",
                               "sample": "std::sort of the same %d keys (oracle, -O2), %.2f s" % (n, wall),
                               "matches": bool(np.array_equal(k2, want))}
    return out


def verify(gt, mix, res, src, arr):
    """Every root of the mix against the oracle, exactly: fib and n-queens
    values and task counts, and every cilksort segment byte-identical to a
    plain sort of its input (the check of examples/cilksort/cilksort.cu:225-258,
    h == gold).  The segmented sort runs on the device: each key is tagged
    with its segment index in the high 32 bits, so one sort of the tagged keys
    sorts every segment in place."""
    import torch
    from tests import oracle_lib as orc
    ok = all(r.status == gt.ROOT_DONE for r in res)
    for i, r in enumerate(res):
        k, p = int(mix.kind[i]), int(mix.param[i])
        if k == 0:
            ok &= r.value == orc.fib(p) and r.tasks == orc.fib_tasks(p, 0)
        elif k == 1:
            ok &= r.value == orc.nq(p) and r.tasks == orc.nq_tasks(p, p - 1)
    nk = mix.total_keys
    if nk:
        sizes = torch.from_numpy(np.diff(mix.offsets)).cuda()
        seg = torch.repeat_interleave(torch.arange(mix.n, device="cuda", dtype=torch.int64), sizes)
        tagged = (seg << 32) | (src[:nk].long() + (1 << 31))
        del seg
        want = (torch.sort(tagged).values & 0xFFFFFFFF) - (1 << 31)
        del tagged
        ok &= bool(torch.equal(want.int(), arr[:nk]))
        del want
        torch.cuda.empty_cache()
    return bool(ok)


def measure_per_root(gt, roots, res_batch, batched_value, tuned_overrides):
    """The plain per-root baseline: gtap_reset-style relaunch per root
    (gtap_launch_per_root), one pass over the mix, under the better of the
    library defaults and the batch-tuned configuration."""
    import torch
    best = None
    for label, ov in (("library defaults", {}), ("batch-tuned", dict(tuned_overrides))):
        gt.gtap_finalize()
        gt.gtap_initialize(gt.default_config(**ov))
        gt.launch(roots[:64], per_root=True)          # warm
        torch.cuda.synchronize()
        p0 = time.perf_counter()
        res_pr, st_pr = gt.launch(roots, per_root=True)
        torch.cuda.synchronize()
        pr_s = time.perf_counter() - p0
        ok = all(a.value == b.value and a.status == b.status and a.tasks == b.tasks
                 for a, b in zip(res_pr, res_batch))
        tps = sum(r.tasks for r in res_pr) / pr_s
        e = {"config": label, "tasks_per_s": tps, "s_per_step": pr_s, "kernel_ms_sum": st_pr.kernel_ms,
             "results_match": ok}
        if best is None or tps > best["tasks_per_s"]:
            best = e
    gt.gtap_finalize()
    best["speedup_batched_vs_per_root"] = batched_value / best["tasks_per_s"]
    return best


def measure_reference_gpu(gt, reps=12):
    """fib(30) and fib(34) with serial cutoff 12 on the reference GTaP GPU
    build (oracle/_ref/fib_ref, fib_ref_c12: the reference runtime compiled
    from its own headers with the hand-lowered fib, at its evaluation
    geometry), beside this runtime's built-in fib (library defaults and the
    autotuned configuration) and the pragma program lowered by
    gtap_b200.lower in both result schemes.  Each time is the median CUDA-event
    time of the persistent launch over `reps` launches (the first dropped);
    every run's result is checked."""
    import subprocess as sp
    from tests import oracle_lib as orc
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    pragma_dir = os.path.join(ROOT, "tests", "pragma", "bin")

    def run_exe(exe, n, cutoff):
        r = sp.run([exe, str(n), str(cutoff), str(reps)], capture_output=True, text=True, timeout=120)
        if r.returncode != 0:
            return None, "exit %d" % r.returncode
        d = json.loads(r.stdout.strip().splitlines()[-1])
        vals = d.get("results", [d.get("result")])
        if any(v != orc.fib(n) for v in vals) or d.get("error_code", 0) != 0:
            return None, "wrong result"
        return statistics.median(d["ms"][1:]), None

    out = {}
    for name, n, cutoff, ref_exe, tuned in (("fib30", 30, 0, "fib_ref", "b200_fib30.json"),
                                            ("fib34_cutoff12", 34, 12, "fib_ref_c12", "b200_fib34c12.json")):
        e = {"ms": {}, "notes": {}}
        exe = os.path.join(ref_dir, ref_exe)
        if os.path.exists(exe):
            ms, err = run_exe(exe, n, cutoff)
            e["ms"]["reference_build"] = ms
            if err:
                e["notes"]["reference_build"] = err
        else:
            e["notes"]["reference_build"] = "not built (oracle/Makefile ref-gpu needs the reference sources)"
        for label, ov in (("builtin_defaults", {}),
                          ("builtin_tuned", load_tuned(os.path.join(ROOT, "gtap_b200", "tuned", tuned)))):
            gt.gtap_initialize(gt.default_config(**ov))
            try:
                ms = []
                for _ in range(reps):
                    res, st = gt.launch([gt.fib_root(n, cutoff)])
                    assert res[0].value == orc.fib(n) and res[0].tasks == orc.fib_tasks(n, cutoff)
                    ms.append(st.kernel_ms)
                e["ms"][label] = statistics.median(ms[1:])
            finally:
                gt.gtap_finalize()
        for label, b in (("lowered_retain", "fib_pragma"), ("lowered_parent", "fib_pragma_parent")):
            exe = os.path.join(pragma_dir, b)
            if os.path.exists(exe):
                ms, err = run_exe(exe, n, cutoff)
                e["ms"][label] = ms
                if err:
                    e["notes"][label] = err
        ref_ms = e["ms"].get("reference_build")
        if ref_ms:
            e["speedup_vs_reference_build"] = {k: ref_ms / v for k, v in e["ms"].items()
                                               if v and k != "reference_build"}
        if not e["notes"]:
            del e["notes"]
        out[name] = e
    return out


def measure_published_configs(gt, reps=5):
    """The configurations the reference publishes numbers for (GH200,
    evaluation/2-comparison/*/..._performance_results.csv), on this B200:
    n-queens(13) with the reference program's cutoff depth 7 (gtap_nq.cu:66),
    and thread-mode cilksort (cutoffs 64/256, gtap_cilksort.cu:11-12) of 10^7,
    5*10^7 and 10^8 std::mt19937(42) keys standing in for gen_vector files.
    Median CUDA-event kernel time; every result checked (the sorted keys
    against a plain sort of the same keys on the device)."""
    import torch
    from tests import oracle_lib as orc
    out = {}
    gt.gtap_initialize(gt.default_config())
    try:
        ms = []
        for _ in range(reps + 1):
            res, st = gt.launch([gt.nq_root(13, 7)])
            assert res[0].value == orc.nq(13) and res[0].tasks == orc.nq_tasks(13, 7)
            ms.append(st.kernel_ms)
        m = statistics.median(ms[1:])
        out["nq13_cutoff7"] = {"ms": m, "tasks": int(res[0].tasks), "published_gh200_ms": 0.8505,
                               "published_source": "evaluation/2-comparison/nq/nq_performance_results.csv:14",
                               "gh200_over_b200": 0.8505 / m}
        for n, pub, line in ((10 ** 7, 10.217, 8), (5 * 10 ** 7, 36.962, 10), (10 ** 8, 82.1875, 11)):
            keys = orc.keys(42, n)
            src = torch.from_numpy(keys).cuda()
            arr = torch.empty_like(src)
            tmp = torch.empty_like(src)
            root = gt.cilksort_root(src.data_ptr(), arr.data_ptr(), tmp.data_ptr(), n, 64, 256)
            ms = []
            for _ in range(reps + 1):
                res, st = gt.launch([root])
                ms.append(st.kernel_ms)
            ok = res[0].status == gt.ROOT_DONE and bool(torch.equal(arr, torch.sort(src).values))
            m = statistics.median(ms[1:])
            out["cilksort_thread_%d" % n] = {"ms": m, "keys_per_s": n / (m / 1e3), "sorted_equals_plain_sort": ok,
                                             "published_gh200_ms": pub, "gh200_over_b200": pub / m,
                                             "published_source": "evaluation/2-comparison/cilksort/"
                                                                 "cilksort_performance_results.csv:%d" % line}
            del src, arr, tmp
            torch.cuda.empty_cache()
    finally:
        gt.gtap_finalize()
    out["note"] = "published numbers are GH200 (sm_90): context for the same configurations, not a ratio claimed"
    return out


def measure_single_roots(gt, reps=3):
    """One root per launch, library defaults: asynchronous BFS from the
    highest-degree vertex of R-MAT graphs (scale 16/18/20, edge factor 16,
    the serve workload's graphs) and int64 sums over unbalanced binary trees
    (2^18 / 2^20 nodes).  BFS reports GTEPS = CSR edges / kernel time (every
    edge is scanned once per relaxation of its source); depths are checked
    against the oracle's queue BFS, sums exactly."""
    import torch
    from tests import oracle_lib as orc
    out = {"bfs": [], "treesum": []}
    gt.gtap_initialize(gt.default_config())
    try:
        for s in (16, 18, 20):
            row, col = gt.gen_rmat(s, 16, 1000 + s)
            src = gt.max_degree_vertex(row)
            drow, dcol = torch.from_numpy(row).cuda(), torch.from_numpy(col).cuda()
            nv = len(row) - 1
            depth = torch.empty(nv, dtype=torch.int32, device="cuda")
            root = gt.bfs_root(drow.data_ptr(), dcol.data_ptr(), depth.data_ptr(), nv, src, 32)
            ms, tasks = [], 0
            for _ in range(reps + 1):
                depth.fill_(0x3f3f3f3f)
                torch.cuda.synchronize()
                res, st = gt.launch([root])
                ms.append(st.kernel_ms)
                tasks = int(res[0].tasks)
            ok = bool(np.array_equal(depth.cpu().numpy(), orc.bfs(row, col, src)))
            m = statistics.median(ms[1:])
            out["bfs"].append({"scale": s, "vertices": nv, "edges": len(col), "ms": m,
                               "gteps": len(col) / (m / 1e3) / 1e9, "tasks": tasks, "depths_ok": ok})
        for n in (1 << 18, 1 << 20):
            left, right, value, size = gt.gen_tree(n, 2000 + n)
            arrs = [torch.from_numpy(a).cuda() for a in (left, right, value, size)]
            ms = []
            for _ in range(reps + 1):
                res, st = gt.launch([gt.treesum_root(*[a.data_ptr() for a in arrs], n, 0, 32)])
                ms.append(st.kernel_ms)
            m = statistics.median(ms[1:])
            out["treesum"].append({"nodes": n, "ms": m, "tasks": int(res[0].tasks),
                                   "sum_ok": res[0].value == int(value.astype(np.int64).sum())})
    finally:
        gt.gtap_finalize()
    return out


def measure_reference_per_root(gt, mix, overrides, reps=6):
    """The plain per-root baseline with the reference GTaP build itself, for
    the mix's fib roots (the reference build of fib is the one that runs
    correctly here): each distinct n timed by oracle/_ref/fib_ref (the
    reference runtime, gtap_reset + one launch per run, CUDA events around
    the launch, so the reset is not even counted), times the number of roots
    with that n; against the same fib roots batched in one launch of this
    runtime with the mix's configuration."""
    import subprocess as sp
    from tests import oracle_lib as orc
    exe = os.path.join(ROOT, "oracle", "_ref", "fib_ref")
    if not os.path.exists(exe):
        return {"note": "oracle/_ref/fib_ref not built (oracle/Makefile ref-gpu needs the reference sources)"}
    fib_idx = [i for i in range(mix.n) if int(mix.kind[i]) == 0]
    ns = sorted({int(mix.param[i]) for i in fib_idx})
    per_n = {}
    for n in ns:
        r = sp.run([exe, str(n), "0", str(reps)], capture_output=True, text=True, timeout=120)
        d = json.loads(r.stdout.strip().splitlines()[-1])
        if r.returncode != 0 or d.get("result") != orc.fib(n):
            return {"note": "reference build failed on fib(%d)" % n}
        per_n[n] = statistics.median(d["ms"][1:])
    ref_ms = sum(per_n[int(mix.param[i])] for i in fib_idx)
    tasks = sum(orc.fib_tasks(int(mix.param[i]), 0) for i in fib_idx)
    roots = [gt.fib_root(int(mix.param[i]), 0) for i in fib_idx]
    gt.gtap_initialize(gt.default_config(**overrides))
    try:
        ms = []
        for _ in range(4):
            res, st = gt.launch(roots)
            assert all(r.value == orc.fib(int(mix.param[i])) for r, i in zip(res, fib_idx))
            ms.append(st.kernel_ms)
    finally:
        gt.gtap_finalize()
    ours = statistics.median(ms[1:])
    return {"roots": len(fib_idx), "tasks": tasks, "reference_build_per_root_ms": ref_ms,
            "reference_build_tasks_per_s": tasks / (ref_ms / 1e3), "batched_ms": ours,
            "batched_tasks_per_s": tasks / (ours / 1e3), "speedup_batched_vs_reference_per_root": ref_ms / ours,
            "per_n_ms": per_n}


def atomic_view(counters, mix, res, k_ms):
    """L2 atomics the scheduler needs per launch, over the kernel time, against
    the measured peak rate of scattered 32-bit atomic adds with a return value
    (profiles/atomic_peak.json, written by gtap_measure_atomic_rate).  Counted:
    one join-counter decrement per task that has a waiting parent (fib and
    cilksort tasks other than roots), one CAS per own-deque pop and per steal,
    one add per published batch, one per root-counter flush; the per-warp
    batching keeps the last two small."""
    joins = 0
    for i, r in enumerate(res):
        if int(mix.kind[i]) in (0, 2):
            joins += r.tasks - 1
    ops = joins + counters.get("pops", 0) + counters.get("steal_successes", 0) + counters.get("rounds", 0)
    achieved = ops / (k_ms / 1e3) / 1e9
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "profiles", "atomic_peak.json")))["scattered_atom_add_gops"]
    except Exception:
        pass
    return {"bound": "l2_atomics", "achieved": achieved, "unit": "Gatom/s", "ops_per_launch": ops,
            "peak": peak, "frac": (achieved / peak) if peak else None,
            "peak_source": "measured (profiles/atomic_peak.json)" if peak else None}


def measure_e2e(gt, mix, steps, tasks_per_step, world, arr_dev):
    import torch
    pin_src = torch.from_numpy(mix.keys).pin_memory()
    pin_out = torch.empty_like(pin_src).pin_memory()
    pin_tmp = torch.empty(1, dtype=torch.int32)
    roots = []
    base_s, base_o = pin_src.data_ptr(), pin_out.data_ptr()
    for i in range(mix.n):
        k, p = int(mix.kind[i]), int(mix.param[i])
        if k == 0:
            roots.append(gt.fib_root(p, 0))
        elif k == 1:
            roots.append(gt.nq_root(p))
        else:
            o = int(mix.offsets[i]) * 4
            roots.append(gt.cilksort_root(base_s + o, base_o + o, 0, p, SORT_CUTOFF, MERGE_CUTOFF))
    gt.run_host(roots)   # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hin = hout = 0
    for _ in range(steps):
        res, st, hin, hout = gt.run_host(roots)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    n = min(1 << 22, mix.total_keys)
    ok = bool(np.array_equal(pin_out.numpy()[:n], arr_dev[:n].cpu().numpy()))
    ok &= all(r.status == gt.ROOT_DONE for r in res)
    del pin_tmp
    return {"value": world * tasks_per_step * steps / dt, "unit": UNIT, "h2d_bytes_per_step": int(hin),
            "d2h_bytes_per_step": int(hout), "api": "gtap_run_host (pinned host buffers)", "s_per_step": dt / steps,
            "ok": ok}


def traffic_from_profile(key):
    """A figure from the committed ncu summary of DRAM traffic, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(p)).get(key)
    except Exception:
        return None


def scaled_traffic(kernel, alg_bytes):
    """DRAM bytes per launch of a worker kernel: the traffic / algorithmic-bytes
    ratio ncu measured for it on a smaller case of the same roots, times this
    launch's algorithmic bytes (null without a committed measurement)."""
    r = traffic_from_profile(kernel + "_traffic_over_algorithmic")
    return None if r is None else int(alg_bytes * r)


if __name__ == "__main__":
    main()
